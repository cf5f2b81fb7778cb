// ww3-gpu_b200/csrc/abi_va.cu
// The resident-spectrum half of the C ABI (ww_va_*), see va.hpp.
//
// Reference behaviour (ww3-gpu kokkos/src/fortran_iface/resident_shim.cpp, resident_c.hpp):
//  * one context per igrid, bound to the Fortran VA's address and shape on its first call;
//  * host read: DEVICE -> one whole D2H copy, state BOTH; host write: the same, then HOST;
//  * partial read/write of listed columns through a device gather/scatter, state unchanged;
//  * device zeroing of listed columns after a host statement that zeroed them;
//  * ww_va_device: HOST -> one whole H2D copy, state BOTH; write -> DEVICE;
//  * diagnostics WW_KOKKOS_VA_RESIDENT, _CHECK, _POISON, _COUNT read once from the environment.
// Copies move bits and compute nothing.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "va.hpp"
#include "wwb_common.hpp"

namespace wwb {
namespace {

enum class Side { Host, Device, Both };

__global__ void gather_cols_kernel(const float* __restrict__ va, const int* __restrict__ cols,
                                   int ncol, int nspec, float* __restrict__ buf) {
  const size_t n = static_cast<size_t>(ncol) * nspec;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t k = i / nspec, s = i % nspec;
    buf[i] = va[static_cast<size_t>(cols[k]) * nspec + s];
  }
}

__global__ void scatter_cols_kernel(float* __restrict__ va, const int* __restrict__ cols,
                                    int ncol, int nspec, const float* __restrict__ buf) {
  const size_t n = static_cast<size_t>(ncol) * nspec;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t k = i / nspec, s = i % nspec;
    va[static_cast<size_t>(cols[k]) * nspec + s] = buf[i];
  }
}

__global__ void zero_cols_kernel(float* __restrict__ va, const int* __restrict__ cols, int ncol,
                                 int nspec) {
  const size_t n = static_cast<size_t>(ncol) * nspec;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    va[static_cast<size_t>(cols[i / nspec]) * nspec + i % nspec] = 0.0f;
}

int grid_for(size_t n) {
  const size_t b = (n + 255) / 256;
  const size_t cap = static_cast<size_t>(runtime().sm_count > 0 ? runtime().sm_count : 148) * 16;
  return static_cast<int>(std::max<size_t>(1, std::min(b, cap)));
}

struct ColSet {
  std::vector<int> cols;
  int* d_cols = nullptr;
  float* d_buf = nullptr;
  std::vector<float> h_buf;
  void free_dev() {
    if (d_cols) cudaFree(d_cols);
    if (d_buf) cudaFree(d_buf);
    d_cols = nullptr;
    d_buf = nullptr;
  }
};

struct Ctx {
  float* host = nullptr;
  int nspec = 0, nsealm = -1;
  float* d = nullptr;
  Side side = Side::Host;
  std::vector<ColSet> sets;  // most recent first
  std::vector<float> snap;   // WW_KOKKOS_VA_CHECK: host bits at the last sync
  bool snap_ok = false;
  size_t count() const { return static_cast<size_t>(nspec) * static_cast<size_t>(nsealm + 1); }
  size_t bytes() const { return count() * sizeof(float); }
};
constexpr size_t kMaxColSets = 8;

std::map<int, Ctx>& grids() {
  static auto* m = new std::map<int, Ctx>();
  return *m;
}

struct Counts {
  long long h2d = 0, d2h = 0, host_reads = 0, host_writes = 0, device_calls = 0;
  long long part_calls = 0, part_d2h = 0, part_cols = 0;
  long long zero_calls = 0, zero_launches = 0, zero_cols = 0, zero_checks = 0;
  long long wrote_calls = 0, wrote_h2d = 0, wrote_cols = 0;
  long long va_checks = 0, poisons = 0;
  double h2d_bytes = 0, d2h_bytes = 0, spectrum_bytes = 0, part_bytes = 0, wrote_bytes = 0;
};
Counts g_n;
bool g_report_registered = false;

bool env_one(const char* n) {
  const char* v = std::getenv(n);
  return v != nullptr && std::strcmp(v, "1") == 0;
}
bool resident_diag() {
  static const bool on = env_one("WW_KOKKOS_VA_RESIDENT");
  return on;
}
bool check_diag() {
  static const bool on = env_one("WW_KOKKOS_VA_CHECK");
  return on;
}
bool poison_diag() {
  static const bool on = env_one("WW_KOKKOS_VA_POISON");
  return on;
}
bool count_diag() {
  static const bool on = env_one("WW_KOKKOS_VA_COUNT");
  return on;
}

void say(const char* what) { std::fprintf(stderr, "ww_b200: %s\n", what); }

Ctx* bind(int igrid, float* va, int nspec, int nsealm) {
  if (va == nullptr || nspec <= 0 || nsealm < 0) {
    say("ww_va: a null VA or a negative extent");
    return nullptr;
  }
  if (!g_report_registered && count_diag()) {
    std::atexit(ww_va_report);
    g_report_registered = true;
  }
  Ctx& c = grids()[igrid];
  if (c.host == nullptr) {
    c.host = va;
    c.nspec = nspec;
    c.nsealm = nsealm;
    g_n.spectrum_bytes += static_cast<double>(c.bytes());
    return &c;
  }
  if (c.host != va || c.nspec != nspec || c.nsealm != nsealm) {
    std::fprintf(stderr,
                 "ww_b200: ww_va: grid %d's VA moved or changed shape (%p %d x 0:%d, bound %p "
                 "%d x 0:%d); the resident spectrum supports one VA per grid\n",
                 igrid, static_cast<void*>(va), nspec, nsealm, static_cast<void*>(c.host),
                 c.nspec, c.nsealm);
    return nullptr;
  }
  return &c;
}

void snapshot(Ctx& c) {
  if (!check_diag()) return;
  c.snap.assign(c.host, c.host + c.count());
  c.snap_ok = true;
}

long long cols_differ(const Ctx& c, const float* p) {
  const size_t ns = static_cast<size_t>(c.nspec);
  long long bad = 0;
  for (int j = 0; j <= c.nsealm; ++j)
    if (std::memcmp(p + j * ns, c.snap.data() + j * ns, ns * sizeof(float)) != 0) ++bad;
  return bad;
}

int check(Ctx& c, int igrid, const char* where) {
  if (!check_diag() || !c.snap_ok || c.side == Side::Host) return WW_KOKKOS_OK;
  ++g_n.va_checks;
  const long long host_bad = cols_differ(c, c.host);
  if (host_bad != 0) {
    std::fprintf(stderr,
                 "ww_b200: WW_KOKKOS_VA_CHECK: at %s, %lld columns of the host VA of grid %d "
                 "changed since the last sync, and no host write declared it\n",
                 where, host_bad, igrid);
    return WW_KOKKOS_ERR_KERNEL;
  }
  if (c.side == Side::Both && c.d != nullptr) {
    std::vector<float> h(c.count());
    WWB_CHECK(cudaMemcpy(h.data(), c.d, c.bytes(), cudaMemcpyDeviceToHost));
    const long long dev_bad = cols_differ(c, h.data());
    if (dev_bad != 0) {
      std::fprintf(stderr,
                   "ww_b200: WW_KOKKOS_VA_CHECK: at %s, %lld columns of d_va of grid %d differ "
                   "from the host VA while the state says both copies are equal\n",
                   where, dev_bad, igrid);
      return WW_KOKKOS_ERR_KERNEL;
    }
  }
  return WW_KOKKOS_OK;
}

void allocate(Ctx& c) {
  if (c.d != nullptr) return;
  WWB_CHECK(cudaMalloc(&c.d, c.bytes()));
}

void h2d(Ctx& c) {
  allocate(c);
  timers::Region t("va.h2d");
  WWB_CHECK(cudaMemcpy(c.d, c.host, c.bytes(), cudaMemcpyHostToDevice));
  ++g_n.h2d;
  g_n.h2d_bytes += static_cast<double>(c.bytes());
  c.side = Side::Both;
  snapshot(c);
}

void d2h(Ctx& c) {
  timers::Region t("va.d2h");
  WWB_CHECK(cudaDeviceSynchronize());  // kernels on other streams wrote d_va
  WWB_CHECK(cudaMemcpy(c.host, c.d, c.bytes(), cudaMemcpyDeviceToHost));
  ++g_n.d2h;
  g_n.d2h_bytes += static_cast<double>(c.bytes());
  c.side = Side::Both;
  snapshot(c);
}

int host_sync(int igrid, float* va, int nspec, int nsealm, bool write) {
  timers::Region t("va.host.call");
  Ctx* c = bind(igrid, va, nspec, nsealm);
  if (c == nullptr) return WW_KOKKOS_ERR_BAD_SHAPE;
  if (const int rc = check(*c, igrid, write ? "a host write" : "a host read"); rc != WW_KOKKOS_OK)
    return rc;
  if (resident_diag()) {
    if (!runtime().ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
    if (c->side == Side::Host) h2d(*c);
    d2h(*c);
  } else if (c->side == Side::Device) {
    d2h(*c);
  }
  if (write) {
    c->side = Side::Host;
    c->snap_ok = false;
  }
  return WW_KOKKOS_OK;
}

/// Sorted, deduplicated column list, or false when a column is outside 0..nsealm.
bool sorted_cols(int ncol, const int* cols, int nsealm, std::vector<int>& want) {
  want.assign(cols, cols + ncol);
  std::sort(want.begin(), want.end());
  want.erase(std::unique(want.begin(), want.end()), want.end());
  return want.empty() || (want.front() >= 0 && want.back() <= nsealm);
}

ColSet& col_set(Ctx& c, const std::vector<int>& want) {
  auto hit = std::find_if(c.sets.begin(), c.sets.end(),
                          [&](const ColSet& s) { return s.cols == want; });
  if (hit != c.sets.end()) {
    std::rotate(c.sets.begin(), hit, hit + 1);
    return c.sets.front();
  }
  ColSet s;
  s.cols = want;
  const size_t n = want.size();
  WWB_CHECK(cudaMalloc(&s.d_cols, n * sizeof(int)));
  WWB_CHECK(cudaMemcpy(s.d_cols, want.data(), n * sizeof(int), cudaMemcpyHostToDevice));
  WWB_CHECK(cudaMalloc(&s.d_buf, n * static_cast<size_t>(c.nspec) * sizeof(float)));
  s.h_buf.resize(n * static_cast<size_t>(c.nspec));
  if (c.sets.size() >= kMaxColSets) {
    c.sets.back().free_dev();
    c.sets.pop_back();
  }
  c.sets.insert(c.sets.begin(), std::move(s));
  return c.sets.front();
}

int host_read_cols(int igrid, float* va, int nspec, int nsealm, int ncol, const int* cols) {
  timers::Region t("va.host.cols");
  Ctx* c = bind(igrid, va, nspec, nsealm);
  if (c == nullptr) return WW_KOKKOS_ERR_BAD_SHAPE;
  if (ncol < 0 || (ncol > 0 && cols == nullptr)) return WW_KOKKOS_ERR_BAD_SHAPE;
  std::vector<int> want;
  if (!sorted_cols(ncol, cols, nsealm, want)) {
    say("ww_va_host_read_cols: a column outside 0..NSEALM");
    return WW_KOKKOS_ERR_BAD_SHAPE;
  }
  if (const int rc = check(*c, igrid, "a partial host read"); rc != WW_KOKKOS_OK) return rc;
  if (resident_diag()) {
    if (!runtime().ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
    if (c->side == Side::Host) h2d(*c);
  } else if (c->side != Side::Device) {
    return WW_KOKKOS_OK;
  }
  if (want.empty()) return WW_KOKKOS_OK;
  const int n = static_cast<int>(want.size());
  ColSet& cs = col_set(*c, want);
  const size_t ns = static_cast<size_t>(nspec);
  {
    timers::Region tc("va.d2h.cols");
    WWB_CHECK(cudaDeviceSynchronize());
    gather_cols_kernel<<<grid_for(ns * n), 256>>>(c->d, cs.d_cols, n, nspec, cs.d_buf);
    WWB_CHECK(cudaGetLastError());
    WWB_CHECK(cudaMemcpy(cs.h_buf.data(), cs.d_buf, ns * n * sizeof(float),
                         cudaMemcpyDeviceToHost));
  }
  for (int k = 0; k < n; ++k)
    std::memcpy(c->host + cs.cols[k] * ns, cs.h_buf.data() + k * ns, ns * sizeof(float));
  if (c->snap_ok)
    for (int k = 0; k < n; ++k)
      std::memcpy(c->snap.data() + cs.cols[k] * ns, cs.h_buf.data() + k * ns, ns * sizeof(float));
  ++g_n.part_d2h;
  g_n.part_cols += n;
  g_n.part_bytes += static_cast<double>(ns * n * sizeof(float));
  return WW_KOKKOS_OK;
}

int host_wrote_cols(int igrid, float* va, int nspec, int nsealm, int ncol, const int* cols) {
  timers::Region t("va.host.wcols");
  Ctx* c = bind(igrid, va, nspec, nsealm);
  if (c == nullptr) return WW_KOKKOS_ERR_BAD_SHAPE;
  if (ncol < 0 || (ncol > 0 && cols == nullptr)) return WW_KOKKOS_ERR_BAD_SHAPE;
  std::vector<int> want;
  if (!sorted_cols(ncol, cols, nsealm, want)) {
    say("ww_va_host_wrote_cols: a column outside 0..NSEALM");
    return WW_KOKKOS_ERR_BAD_SHAPE;
  }
  const size_t ns = static_cast<size_t>(nspec);
  if (c->snap_ok)
    for (const int j : want)
      std::memcpy(c->snap.data() + j * ns, c->host + j * ns, ns * sizeof(float));
  if (const int rc = check(*c, igrid, "a partial host write"); rc != WW_KOKKOS_OK) return rc;
  if (c->side == Side::Host || want.empty()) {
    if (resident_diag() && c->side == Side::Host) {
      if (!runtime().ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
      h2d(*c);
    }
    return WW_KOKKOS_OK;
  }
  if (!runtime().ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
  const int n = static_cast<int>(want.size());
  ColSet& cs = col_set(*c, want);
  for (int k = 0; k < n; ++k)
    std::memcpy(cs.h_buf.data() + k * ns, c->host + cs.cols[k] * ns, ns * sizeof(float));
  {
    timers::Region tc("va.h2d.cols");
    WWB_CHECK(cudaDeviceSynchronize());
    WWB_CHECK(cudaMemcpy(cs.d_buf, cs.h_buf.data(), ns * n * sizeof(float),
                         cudaMemcpyHostToDevice));
    scatter_cols_kernel<<<grid_for(ns * n), 256>>>(c->d, cs.d_cols, n, nspec, cs.d_buf);
    WWB_CHECK(cudaGetLastError());
    WWB_CHECK(cudaDeviceSynchronize());
  }
  ++g_n.wrote_h2d;
  g_n.wrote_cols += n;
  g_n.wrote_bytes += static_cast<double>(ns * n * sizeof(float));
  if (resident_diag()) d2h(*c);
  return WW_KOKKOS_OK;
}

int device_zero_cols(int igrid, float* va, int nspec, int nsealm, int ncol, const int* cols) {
  timers::Region t("va.zero.cols");
  Ctx* c = bind(igrid, va, nspec, nsealm);
  if (c == nullptr) return WW_KOKKOS_ERR_BAD_SHAPE;
  if (ncol < 0 || (ncol > 0 && cols == nullptr)) return WW_KOKKOS_ERR_BAD_SHAPE;
  for (int k = 0; k < ncol; ++k)
    if (cols[k] < 0 || cols[k] > nsealm) {
      say("ww_va_device_zero_cols: a column outside 0..NSEALM");
      return WW_KOKKOS_ERR_BAD_SHAPE;
    }
  if (c->side == Side::Host) return WW_KOKKOS_OK;
  if (!runtime().ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
  const size_t ns = static_cast<size_t>(nspec);
  if (ncol > 0) {
    int* dc = nullptr;
    WWB_CHECK(cudaMalloc(&dc, ncol * sizeof(int)));
    WWB_CHECK(cudaMemcpy(dc, cols, ncol * sizeof(int), cudaMemcpyHostToDevice));
    WWB_CHECK(cudaDeviceSynchronize());
    zero_cols_kernel<<<grid_for(ns * ncol), 256>>>(c->d, dc, ncol, nspec);
    const cudaError_t e = cudaGetLastError();
    cudaDeviceSynchronize();
    cudaFree(dc);
    WWB_CHECK(e);
    ++g_n.zero_launches;
    g_n.zero_cols += ncol;
  }
  if (c->snap_ok)
    for (int k = 0; k < ncol; ++k) std::fill_n(c->snap.data() + cols[k] * ns, ns, 0.0f);
  if (resident_diag()) {
    std::vector<float> back(c->count());
    WWB_CHECK(cudaMemcpy(back.data(), c->d, c->bytes(), cudaMemcpyDeviceToHost));
    long long bad = 0;
    for (int j = 0; j <= c->nsealm; ++j)
      if (std::memcmp(back.data() + j * ns, c->host + j * ns, ns * sizeof(float)) != 0) ++bad;
    ++g_n.zero_checks;
    if (bad != 0) {
      std::fprintf(stderr,
                   "ww_b200: ww_va_device_zero_cols: %lld columns of VA differ between the host "
                   "and the device after the update of grid %d\n",
                   bad, igrid);
      return WW_KOKKOS_ERR_KERNEL;
    }
  }
  return WW_KOKKOS_OK;
}

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc& e) {
    say(e.what());
    return WW_KOKKOS_ERR_RUNTIME;
  } catch (const std::exception& e) {
    say(e.what());
    return WW_KOKKOS_ERR_KERNEL;
  }
}

}  // namespace

int va_device(int igrid, float* va, int nspec, int nsealm, float** d_va) {
  return guarded([&]() {
    if (!runtime().ready) return static_cast<int>(WW_KOKKOS_ERR_NOT_INITIALISED);
    Ctx* c = bind(igrid, va, nspec, nsealm);
    if (c == nullptr) return static_cast<int>(WW_KOKKOS_ERR_BAD_SHAPE);
    if (const int rc = check(*c, igrid, "a kernel's sync"); rc != WW_KOKKOS_OK) return rc;
    ++g_n.device_calls;
    if (c->side == Side::Host) h2d(*c);
    *d_va = c->d;
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

void va_device_written(int igrid) {
  auto it = grids().find(igrid);
  if (it == grids().end() || it->second.d == nullptr) return;
  Ctx& c = it->second;
  c.side = Side::Device;
  if (poison_diag()) {
    const uint32_t bits = 0x7FC0BAD0u;  // a quiet NaN: a host read that skipped its sync shows
    float nan;
    std::memcpy(&nan, &bits, sizeof nan);
    std::fill_n(c.host, c.count(), nan);
    c.snap_ok = false;
    ++g_n.poisons;
  }
}

void release_va_contexts() {
  for (auto& [igrid, c] : grids()) {
    if (c.side == Side::Device)
      std::fprintf(stderr, "ww_b200: VA of grid %d was still newer on the device at finalize\n",
                   igrid);
    for (auto& s : c.sets) s.free_dev();
    if (c.d) cudaFree(c.d);
    c.d = nullptr;
  }
  grids().clear();
}

}  // namespace wwb

using namespace wwb;

extern "C" {

int ww_va_host_read(int igrid, float* va, int nspec, int nsealm) {
  ++g_n.host_reads;
  return guarded([&]() { return host_sync(igrid, va, nspec, nsealm, false); });
}

int ww_va_host_write(int igrid, float* va, int nspec, int nsealm) {
  ++g_n.host_writes;
  return guarded([&]() { return host_sync(igrid, va, nspec, nsealm, true); });
}

int ww_va_host_read_cols(int igrid, float* va, int nspec, int nsealm, int ncol,
                         const int* cols) {
  ++g_n.part_calls;
  return guarded([&]() { return host_read_cols(igrid, va, nspec, nsealm, ncol, cols); });
}

int ww_va_host_wrote_cols(int igrid, float* va, int nspec, int nsealm, int ncol,
                          const int* cols) {
  ++g_n.wrote_calls;
  return guarded([&]() { return host_wrote_cols(igrid, va, nspec, nsealm, ncol, cols); });
}

int ww_va_host_update(int igrid, float* va, int nspec, int nsealm) {
  ++g_n.zero_calls;
  return guarded([&]() {
    if (!resident_diag()) {
      Ctx* c = bind(igrid, va, nspec, nsealm);
      if (c == nullptr) return static_cast<int>(WW_KOKKOS_ERR_BAD_SHAPE);
      return check(*c, igrid, "a host update");
    }
    ++g_n.host_reads;
    return host_sync(igrid, va, nspec, nsealm, false);
  });
}

int ww_va_device_zero_cols(int igrid, float* va, int nspec, int nsealm, int ncol,
                           const int* cols) {
  return guarded([&]() { return device_zero_cols(igrid, va, nspec, nsealm, ncol, cols); });
}

int ww_va_device(int igrid, int write) {
  return guarded([&]() {
    auto it = grids().find(igrid);
    if (it == grids().end() || !runtime().ready)
      return static_cast<int>(WW_KOKKOS_ERR_NOT_INITIALISED);
    Ctx& c = it->second;
    if (const int rc = check(c, it->first, "a kernel's sync"); rc != WW_KOKKOS_OK) return rc;
    ++g_n.device_calls;
    if (c.side == Side::Host) h2d(c);
    if (write != 0) c.side = Side::Device;
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

void* ww_va_device_ptr(int igrid) {
  auto it = grids().find(igrid);
  return it == grids().end() ? nullptr : static_cast<void*>(it->second.d);
}

int ww_va_state(int igrid) {
  auto it = grids().find(igrid);
  if (it == grids().end()) return -1;
  return static_cast<int>(it->second.side);
}

void ww_va_report(void) {
  constexpr double mb = 1.0e6;
  std::fprintf(stderr,
               "ww_b200: VA: H2D %lld (%.2f MB), D2H %lld (%.2f MB); host reads %lld, host writes "
               "%lld, device syncs %lld; partial reads %lld, of which %lld copied %lld columns "
               "(%.4f MB); spectrum %.2f MB%s\n",
               g_n.h2d, g_n.h2d_bytes / mb, g_n.d2h, g_n.d2h_bytes / mb, g_n.host_reads,
               g_n.host_writes, g_n.device_calls, g_n.part_calls, g_n.part_d2h, g_n.part_cols,
               g_n.part_bytes / mb, g_n.spectrum_bytes / mb,
               resident_diag() ? " (WW_KOKKOS_VA_RESIDENT=1: both copies at every host call)" : "");
  std::fprintf(stderr, "ww_b200: VA host-to-device copies: %lld\n", g_n.h2d);
  std::fprintf(stderr, "ww_b200: VA device-to-host copies: %lld\n", g_n.d2h);
  std::fprintf(stderr, "ww_b200: VA host sync calls: %lld\n", g_n.host_reads + g_n.host_writes);
  std::fprintf(stderr, "ww_b200: VA device sync calls: %lld\n", g_n.device_calls);
  std::fprintf(stderr, "ww_b200: VA partial host reads: %lld\n", g_n.part_calls);
  std::fprintf(stderr, "ww_b200: VA partial device-to-host copies: %lld\n", g_n.part_d2h);
  std::fprintf(stderr, "ww_b200: VA partial columns copied: %lld\n", g_n.part_cols);
  std::fprintf(stderr, "ww_b200: VA partial host writes: %lld\n", g_n.wrote_calls);
  std::fprintf(stderr, "ww_b200: VA partial host-to-device copies: %lld\n", g_n.wrote_h2d);
  std::fprintf(stderr, "ww_b200: VA partial columns stored: %lld (%.4f MB)\n", g_n.wrote_cols,
               g_n.wrote_bytes / mb);
  std::fprintf(stderr, "ww_b200: VA host updates repeated on the device: %lld\n", g_n.zero_calls);
  std::fprintf(stderr, "ww_b200: VA device zeroing launches: %lld\n", g_n.zero_launches);
  std::fprintf(stderr, "ww_b200: VA device columns zeroed: %lld\n", g_n.zero_cols);
  std::fprintf(stderr, "ww_b200: VA zeroing checks run: %lld\n", g_n.zero_checks);
  std::fprintf(stderr, "ww_b200: VA consistency checks run (WW_KOKKOS_VA_CHECK): %lld\n",
               g_n.va_checks);
  std::fprintf(stderr, "ww_b200: VA host copies poisoned (WW_KOKKOS_VA_POISON): %lld\n",
               g_n.poisons);
}

}  // extern "C"
