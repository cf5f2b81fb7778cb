// ww3-gpu_b200/csrc/wwb_common.hpp
// Shared plumbing of libww_b200.so: status codes, the error recorder behind the
// ww_*_last_error() entries, and the CUDA error check that turns a failed runtime call into a
// status instead of an exception crossing the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/ww_b200.h"

namespace wwb {

/// One status cell per part (DIA, VA, PR3 ...), like the reference's per-shim atomics
/// (kokkos/src/fortran_iface/snl1_shim.cpp:92-110): a relaxed atomic, one stderr line per failure.
struct Status {
  std::atomic<int> code{WW_KOKKOS_OK};
  void ok() { code.store(WW_KOKKOS_OK, std::memory_order_relaxed); }
  int fail(int c, const char* what) {
    code.store(c, std::memory_order_relaxed);
    std::fprintf(stderr, "ww_b200: %s (code %d)\n", what, c);
    return c;
  }
  int get() const { return code.load(std::memory_order_relaxed); }
};

/// A CUDA runtime failure inside an entry point; caught at the boundary.
struct CudaError : std::runtime_error {
  cudaError_t err;
  CudaError(cudaError_t e, const char* where)
      : std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e)), err(e) {}
};

inline void check(cudaError_t e, const char* where) {
  if (e != cudaSuccess) throw CudaError(e, where);
}

#define WWB_CHECK(call) ::wwb::check((call), #call)

/// Runtime state shared by every part: whether ww_kokkos_init() ran, the device, the
/// library's own stream for the host-pointer entries.
struct Runtime {
  bool ready = false;
  int device = 0;
  cudaStream_t stream = nullptr;   ///< compute stream of the host-pointer entries
  cudaStream_t copy_in = nullptr;  ///< H2D stream of the pipelined host-pointer entries
  cudaStream_t copy_out = nullptr; ///< D2H stream
  int sm_count = 0;
};
Runtime& runtime();

/// WW_KOKKOS_TIMERS=1 region totals (reference kokkos/src/fortran_iface/timers.hpp:1-12): the
/// wall time of "<part>.<phase>" regions, printed at exit, one line per region.
namespace timers {
bool enabled();
void add(const char* name, double seconds);
class Region {
 public:
  explicit Region(const char* name);
  ~Region() { stop(); }
  void stop();
  Region(const Region&) = delete;
  Region& operator=(const Region&) = delete;

 private:
  const char* name_;
  bool on_;
  double t0_ = 0;
};
}  // namespace timers

}  // namespace wwb
