// ww3-gpu_b200/csrc/staging.hpp
// Grow-only device buffers for the host-pointer entries: a numbered slot per argument, kept
// across calls, so a call with the same sizes allocates nothing (the reference keeps its
// staging Views the same way, kokkos/src/fortran_iface/prop3_shim.cpp:60-140).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "wwb_common.hpp"

namespace wwb {

class Staging {
 public:
  ~Staging() { release(); }
  void release() {
    for (auto& s : slots_)
      if (s.ptr) cudaFree(s.ptr);
    slots_.clear();
  }
  /// A device buffer of at least `bytes` in slot `i`.
  void* get(size_t i, size_t bytes) {
    if (slots_.size() <= i) slots_.resize(i + 1);
    Slot& s = slots_[i];
    if (s.bytes < bytes) {
      if (s.ptr) WWB_CHECK(cudaFree(s.ptr));
      s.ptr = nullptr;
      s.bytes = 0;
      WWB_CHECK(cudaMalloc(&s.ptr, bytes ? bytes : 16));
      s.bytes = bytes;
    }
    return s.ptr;
  }
  /// Slot `i` filled with `n` elements from host memory `h` (asynchronously on `st`).
  template <class T>
  T* in(size_t i, const T* h, size_t n, cudaStream_t st) {
    T* d = static_cast<T*>(get(i, n * sizeof(T)));
    if (n) WWB_CHECK(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return d;
  }

 private:
  struct Slot {
    void* ptr = nullptr;
    size_t bytes = 0;
  };
  std::vector<Slot> slots_;
};

}  // namespace wwb
