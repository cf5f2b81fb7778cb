// ww3-gpu_b200/csrc/abi_snl1.cpp
// The W3SNL1 half of the C ABI: per-grid contexts (INSNL1 tables on the device), the
// host-pointer entry ww_snl1 with its copies pipelined against the kernel, and the
// device-resident entry ww_snl1_device.
//
// Reference: ww3-gpu kokkos/src/fortran_iface/snl1_shim.cpp:254-415 (validation order, status
// codes, "nothing written on a validation failure", npts == 0 no-op, one context per igrid in a
// never-destroyed map) and ww_kokkos_c.hpp:81-133.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "autotune.hpp"
#include "snl1_kernel.cuh"
#include "snl1_tables.hpp"
#include "step.hpp"
#include "wwb_common.hpp"

namespace wwb {
namespace {

/// A device allocation owned by a context.
template <class T>
struct DevBuf {
  T* ptr = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  void reset() {
    free_table(ptr);
    ptr = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    reset();
    if (count == 0) return;
    WWB_CHECK(cudaMalloc(&ptr, count * sizeof(T)));
    n = count;
  }
  void upload(const T* host, size_t count) {
    alloc(count);
    if (count) WWB_CHECK(cudaMemcpy(ptr, host, count * sizeof(T), cudaMemcpyHostToDevice));
  }
};

/// Host-pointer pipeline: kSlots chunks in flight, each on its own stream, so the H2D copy of
/// one chunk, the kernel of the next and the D2H copy of a third overlap.
constexpr int kSlots = 3;
constexpr int kChunkPoints = 8192;

struct Slot {
  cudaStream_t stream = nullptr;
  DevBuf<float> a, cg, kd, s, d;
};

struct Ctx {
  Snl1Config cfg{};
  int device = -1;  ///< the device current at ww_snl1_init: the tables live there
  std::vector<float> sig_host;
  Snl1Tables tab;
  Snl1Dev dev{};
  int kernel = kSnl1Auto;
  DevBuf<float> sig, af11, af11_row;
  DevBuf<int> ipim, ic, ifrow;
  Slot slots[kSlots];
  int slot_capacity = 0;
  bool ready = false;
  ~Ctx() {
    for (auto& sl : slots)
      if (sl.stream) cudaStreamDestroy(sl.stream);
  }
};

std::map<int, Ctx*>& contexts() {
  static auto* m = new std::map<int, Ctx*>();
  return *m;
}

Status g_status;

void erase(int igrid) {
  auto& m = contexts();
  auto it = m.find(igrid);
  if (it != m.end()) {
    delete it->second;
    m.erase(it);
  }
}

/// Uploads the tables of `c` and fills its kernel parameters.
void publish(Ctx& c) {
  const Snl1Tables& t = c.tab;
  c.ipim.upload(t.ipim.data(), t.ipim.size());
  c.ic.upload(t.ic.data(), t.ic.size());
  c.af11.upload(t.af11.data(), t.af11.size());
  if (t.rowshift) {
    c.ifrow.upload(t.ifrow.data(), t.ifrow.size());
    c.af11_row.upload(t.af11_row.data(), t.af11_row.size());
  }
  Snl1Dev& p = c.dev;
  p = Snl1Dev{};
  p.nk = c.cfg.nk;
  p.nth = c.cfg.nth;
  p.nfr = t.nfr;
  p.nfrhgh = t.nfrhgh;
  p.nfrchg = t.nfrchg;
  p.nspec = t.nspec;
  p.nspecx = t.nspecx;
  p.dal1 = t.dal1;
  p.dal2 = t.dal2;
  p.dal3 = t.dal3;
  for (int j = 0; j < 8; ++j) {
    p.awg[j] = t.awg[j];
    p.swg[j] = t.swg[j];
    p.shift[j] = t.shift[j];
  }
  p.ifrp = t.ifrp;
  p.ifrm = t.ifrm;
  p.snlc1 = c.cfg.snlc1;
  p.kdcon = c.cfg.kdcon;
  p.kdmn = c.cfg.kdmn;
  p.snls1 = c.cfg.snls1;
  p.snls2 = c.cfg.snls2;
  p.snls3 = c.cfg.snls3;
  p.fachfe = c.cfg.fachfe;
  p.ifrow = c.ifrow.ptr;
  p.af11_row = c.af11_row.ptr;
  p.ipim = c.ipim.ptr;
  p.ic = c.ic.ptr;
  p.af11 = c.af11.ptr;
  c.kernel = !t.rowshift          ? kSnl1Gather
             : snl1_pair_ok(p)    ? kSnl1Pair
             : snl1_band_ok(p)    ? kSnl1Band
                                  : kSnl1RowShift;
}

/// The kernel `which` asks for, or -1 when these tables cannot run it.
int pick_kernel(const Ctx& c, int which) {
  switch (which) {
    case kSnl1Auto:
      return !c.tab.rowshift           ? kSnl1Gather
             : snl1_pair_ok(c.dev)     ? kSnl1Pair
             : snl1_band_ok(c.dev)     ? kSnl1Band
                                       : kSnl1RowShift;
    case kSnl1Gather:
      return kSnl1Gather;
    case kSnl1RowShift:
      return c.tab.rowshift ? kSnl1RowShift : -1;
    case kSnl1Band:
      return c.tab.rowshift && snl1_band_ok(c.dev) ? kSnl1Band : -1;
    case kSnl1Tile:
      return c.tab.rowshift && snl1_tile_ok(c.dev) ? kSnl1Tile : -1;
    case kSnl1Pair:
      return c.tab.rowshift && snl1_pair_ok(c.dev) ? kSnl1Pair : -1;
    case kSnl1PairGeneral:
      return c.tab.rowshift && snl1_pair_ok(c.dev) ? kSnl1PairGeneral : -1;
    default:
      return -1;
  }
}

int resolve_kernel(const Ctx& c) { return c.kernel; }

/// Common validation of the compute entries; returns the context or nullptr (status set).
Ctx* validate(int igrid, int npts, const void* a, const void* cg, const void* kd, const void* s,
              const void* d, const char* who) {
  auto it = contexts().find(igrid);
  if (it == contexts().end() || !it->second->ready || !runtime().ready) {
    g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_snl1 before ww_snl1_init for this grid");
    return nullptr;
  }
  if (npts < 0) {
    g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1: npts is negative");
    return nullptr;
  }
  if (npts == 0) {
    g_status.ok();
    return nullptr;
  }
  if (!a || !cg || !kd || !s || !d) {
    g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1: null array pointer");
    return nullptr;
  }
  (void)who;
  return it->second;
}

int init_common(int igrid, const Snl1Config& cfg, const float* sig, Snl1Tables&& tab) {
  Ctx* c = new Ctx();
  try {
    c->cfg = cfg;
    c->tab = std::move(tab);
    std::vector<float> h_sig(sig, sig + cfg.nk);
    c->sig.upload(h_sig.data(), h_sig.size());
    c->sig_host = h_sig;
    WWB_CHECK(cudaGetDevice(&c->device));
    publish(*c);
    c->dev.sig = c->sig.ptr;
    for (auto& sl : c->slots) WWB_CHECK(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
    c->ready = true;
  } catch (...) {
    delete c;
    throw;
  }
  contexts()[igrid] = c;
  g_status.ok();
  return WW_KOKKOS_OK;
}

}  // namespace

/// The DIA state of grid igrid for W3SRCE (device tables, row-shift form), or false.
bool snl1_grid_dev(int igrid, Snl1Dev* out) {
  auto it = contexts().find(igrid);
  if (it == contexts().end() || !it->second->ready || !it->second->tab.rowshift) return false;
  *out = it->second->dev;
  return true;
}

/// The configuration and SIG(1:NK) of grid igrid, or false.
bool snl1_grid_config(int igrid, Snl1Config* cfg, std::vector<float>* sig) {
  auto it = contexts().find(igrid);
  if (it == contexts().end() || !it->second->ready) return false;
  *cfg = it->second->cfg;
  *sig = it->second->sig_host;
  return true;
}

void release_snl1_contexts() {
  auto& m = contexts();
  for (auto& kv : m) delete kv.second;
  m.clear();
}

}  // namespace wwb

using namespace wwb;

extern "C" {

int ww_snl1_init(int igrid, int nk, int nth, float xfr, float dth, float lam, float snlc1,
                 float kdcon, float kdmn, float snls1, float snls2, float snls3, float fachfe,
                 const float* sig) {
  try {
    erase(igrid);  // a failure below leaves the grid unconfigured, not half-configured
    if (!runtime().ready)
      return g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_snl1_init before ww_kokkos_init");
    if (nk <= 0 || nth <= 0 || sig == nullptr)
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                           "ww_snl1_init: nk and nth must be > 0 and sig non-null");
    const Snl1Config cfg{nk, nth, xfr, dth, lam, snlc1, kdcon, kdmn, snls1, snls2, snls3, fachfe};
    Snl1Tables tab;
    if (!build_snl1_tables(cfg, sig, tab))
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_init: no extended spectrum");
    return init_common(igrid, cfg, sig, std::move(tab));
  } catch (const std::bad_alloc& e) {
    erase(igrid);
    return g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  } catch (const std::exception& e) {
    erase(igrid);
    return g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  }
}

int ww_snl1_init_tables(int igrid, int nk, int nth, float xfr, float dth, float lam,
                        float snlc1, float kdcon, float kdmn, float snls1, float snls2,
                        float snls3, float fachfe, const float* sig, const int* scal,
                        const float* wts, const int* ipim, const int* ic, const float* af11) {
  try {
    erase(igrid);
    if (!runtime().ready)
      return g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED,
                           "ww_snl1_init_tables before ww_kokkos_init");
    if (nk <= 0 || nth <= 0 || !sig || !scal || !wts || !ipim || !ic || !af11)
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                           "ww_snl1_init_tables: bad extents or null pointer");
    const Snl1Config cfg{nk, nth, xfr, dth, lam, snlc1, kdcon, kdmn, snls1, snls2, snls3, fachfe};
    Snl1Tables t;
    t.nth = nth;
    t.nspec = nk * nth;
    t.nfr = scal[0];
    t.nfrhgh = scal[1];
    t.nfrchg = scal[2];
    t.nspecx = scal[3];
    t.nspecy = scal[4];
    if (t.nfr != nk || t.nfrchg < t.nfr || t.nfrhgh < t.nfrchg || t.nspecx != t.nfrchg * nth ||
        t.nspecy != t.nfrhgh * nth)
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_init_tables: inconsistent sizes");
    t.dal1 = wts[0];
    t.dal2 = wts[1];
    t.dal3 = wts[2];
    for (int j = 0; j < 8; ++j) {
      t.awg[j] = wts[3 + j];
      t.swg[j] = wts[11 + j];
    }
    t.ipim.assign(ipim, ipim + 16 * static_cast<size_t>(t.nspecx));
    t.ic.assign(ic, ic + 16 * static_cast<size_t>(t.nspec));
    t.af11.assign(af11, af11 + t.nspecx);
    // Every entry must address the scratch range the kernels hold: UE slots for the
    // interaction tables, interaction-array slots for IC.
    for (int v : t.ipim)
      if (v + nth < 0 || v + nth >= t.nspecy + nth)
        return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_init_tables: IP/IM out of range");
    for (int v : t.ic)
      if (v + nth < 0 || v + nth >= t.nspecx + nth)
        return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_init_tables: IC out of range");
    derive_rowshift(cfg, t);
    return init_common(igrid, cfg, sig, std::move(t));
  } catch (const std::bad_alloc& e) {
    erase(igrid);
    return g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  } catch (const std::exception& e) {
    erase(igrid);
    return g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  }
}

void ww_snl1(int igrid, int npts, const float* a, const float* cg, const float* kdmean,
             float* s, float* d) {
  try {
    Ctx* c = validate(igrid, npts, a, cg, kdmean, s, d, "ww_snl1");
    if (c == nullptr) return;
    timers::Region t_call("snl1.call");
    const int nspec = c->cfg.nspec(), nk = c->cfg.nk;
    const int chunk = std::min(npts, kChunkPoints);
    if (chunk > c->slot_capacity) {
      for (auto& sl : c->slots) {
        WWB_CHECK(cudaStreamSynchronize(sl.stream));
        sl.a.alloc(static_cast<size_t>(chunk) * nspec);
        sl.cg.alloc(static_cast<size_t>(chunk) * nk);
        sl.kd.alloc(static_cast<size_t>(chunk));
        sl.s.alloc(static_cast<size_t>(chunk) * nspec);
        sl.d.alloc(static_cast<size_t>(chunk) * nspec);
      }
      c->slot_capacity = chunk;
    }
    const int kernel = resolve_kernel(*c);
    int k = 0;
    for (int p0 = 0; p0 < npts; p0 += chunk, ++k) {
      Slot& sl = c->slots[k % kSlots];
      const int n = std::min(chunk, npts - p0);
      const size_t ns = static_cast<size_t>(n) * nspec;
      WWB_CHECK(cudaMemcpyAsync(sl.a.ptr, a + static_cast<size_t>(p0) * nspec, ns * 4,
                                cudaMemcpyHostToDevice, sl.stream));
      WWB_CHECK(cudaMemcpyAsync(sl.cg.ptr, cg + static_cast<size_t>(p0) * nk,
                                static_cast<size_t>(n) * nk * 4, cudaMemcpyHostToDevice,
                                sl.stream));
      WWB_CHECK(cudaMemcpyAsync(sl.kd.ptr, kdmean + p0, static_cast<size_t>(n) * 4,
                                cudaMemcpyHostToDevice, sl.stream));
      launch_snl1(kernel, c->dev, n, sl.a.ptr, sl.cg.ptr, sl.kd.ptr, sl.s.ptr, sl.d.ptr,
                  sl.stream);
      WWB_CHECK(cudaMemcpyAsync(s + static_cast<size_t>(p0) * nspec, sl.s.ptr, ns * 4,
                                cudaMemcpyDeviceToHost, sl.stream));
      WWB_CHECK(cudaMemcpyAsync(d + static_cast<size_t>(p0) * nspec, sl.d.ptr, ns * 4,
                                cudaMemcpyDeviceToHost, sl.stream));
    }
    for (auto& sl : c->slots) WWB_CHECK(cudaStreamSynchronize(sl.stream));
    if (snl1_take_error() != 0) {
      g_status.fail(WW_KOKKOS_ERR_KERNEL, "ww_snl1: a bulk-copy wait of the DIA kernel gave up");
      return;
    }
    g_status.ok();
  } catch (const CudaError& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  } catch (const std::bad_alloc& e) {
    g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

void ww_snl1_device(int igrid, int npts, const float* a, const float* cg, const float* kdmean,
                    float* s, float* d, void* stream) {
  try {
    Ctx* c = validate(igrid, npts, a, cg, kdmean, s, d, "ww_snl1_device");
    if (c == nullptr) return;
    launch_snl1(resolve_kernel(*c), c->dev, npts, a, cg, kdmean, s, d,
                static_cast<cudaStream_t>(stream));
    g_status.ok();
  } catch (const CudaError& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

void ww_snl1_noalloc(int igrid, int npts, const float* a, const float* cg, const float* kdmean,
                     float* s, float* d) {
  try {
    Ctx* c = validate(igrid, npts, a, cg, kdmean, s, d, "ww_snl1_noalloc");
    if (c == nullptr) return;
    const size_t nspec = c->cfg.nspec(), nk = c->cfg.nk, n = static_cast<size_t>(npts);
    auto seg = [](size_t floats) { return (floats + 63) & ~static_cast<size_t>(63); };  // 256 B
    auto need = [&](size_t m) { return 3 * seg(m * nspec) + seg(m * nk) + seg(m); };
    // The static array is per device and picked by the current device; the grid's tables and
    // stream belong to the device of its ww_snl1_init, so the two must be the same.
    int current = -1;
    WWB_CHECK(cudaGetDevice(&current));
    if (current != c->device) {
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                    "ww_snl1_noalloc: the current device is not the one this grid was set up on");
      return;
    }
    const Snl1StaticScratch sc = snl1_static_scratch();  // first call on a device: set-up
    if (need(n) > sc.floats) {
      size_t most = sc.floats / (3 * nspec + nk + 1);
      while (most > 0 && need(most) > sc.floats) --most;
      char msg[200];
      std::snprintf(msg, sizeof msg,
                    "ww_snl1_noalloc: %d points exceed its %zu MiB static scratch (at most %zu "
                    "points of this grid per call)",
                    npts, sc.floats * sizeof(float) >> 20, most);
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, msg);
      return;
    }
    float* const da = sc.base;
    float* const ds = da + seg(n * nspec);
    float* const dd = ds + seg(n * nspec);
    float* const dcg = dd + seg(n * nspec);
    float* const dkd = dcg + seg(n * nk);
    cudaStream_t st = c->slots[0].stream;
    WWB_CHECK(cudaMemsetAsync(sc.err, 0, sizeof(int), st));
    WWB_CHECK(cudaMemcpyAsync(da, a, n * nspec * 4, cudaMemcpyHostToDevice, st));
    WWB_CHECK(cudaMemcpyAsync(dcg, cg, n * nk * 4, cudaMemcpyHostToDevice, st));
    WWB_CHECK(cudaMemcpyAsync(dkd, kdmean, n * 4, cudaMemcpyHostToDevice, st));
    launch_snl1_err(resolve_kernel(*c), c->dev, npts, da, dcg, dkd, ds, dd, sc.err, st);
    WWB_CHECK(cudaMemcpyAsync(s, ds, n * nspec * 4, cudaMemcpyDeviceToHost, st));
    WWB_CHECK(cudaMemcpyAsync(d, dd, n * nspec * 4, cudaMemcpyDeviceToHost, st));
    int flag = 0;
    WWB_CHECK(cudaMemcpyAsync(&flag, sc.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    WWB_CHECK(cudaStreamSynchronize(st));
    if (flag != 0) {
      g_status.fail(WW_KOKKOS_ERR_KERNEL,
                    "ww_snl1_noalloc: a bulk-copy wait of the DIA kernel gave up");
      return;
    }
    g_status.ok();
  } catch (const CudaError& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_snl1_enabled(void) { return ww_kokkos_flag("WW_KOKKOS_SNL1") != 0 ? 1 : 0; }

int ww_snl1_last_error(void) { return g_status.get(); }

int ww_snl1_test_stall(int igrid, int bytes) {
  auto it = contexts().find(igrid);
  if (it == contexts().end() || !it->second->ready) return WW_KOKKOS_ERR_NOT_INITIALISED;
  if (bytes < 0 || bytes > 1024) return WW_KOKKOS_ERR_BAD_SHAPE;
  it->second->dev.stall_tx = bytes;
  return WW_KOKKOS_OK;
}

int ww_snl1_autotune(int igrid) {
  try {
    auto it = contexts().find(igrid);
    if (it == contexts().end() || !it->second->ready) return -1;
    Ctx& c = *it->second;
    std::vector<int> cands;
    for (int k : {kSnl1Pair, kSnl1PairGeneral, kSnl1Band, kSnl1Tile, kSnl1RowShift, kSnl1Gather})
      if (pick_kernel(c, k) == k) cands.push_back(k);
    if (cands.empty()) return -1;
    // 16,384 synthetic points (every point the same smooth spectrum): the DIA's work does not
    // depend on the values, and the batch is large enough to fill every SM many times.
    const int n = 16384;
    const size_t nspec = c.cfg.nspec(), nk = c.cfg.nk;
    std::vector<float> ha(nspec * n), hc(nk * n, 1.5f), hk(n, 3.0f);
    for (size_t i = 0; i < nspec; ++i) ha[i] = 1e-4f * (1.0f + static_cast<float>(i % 37) / 37.0f);
    for (int p = 1; p < n; ++p) std::copy(ha.begin(), ha.begin() + nspec, ha.begin() + p * nspec);
    DevBuf<float> a, cg, kd, s, d;
    a.alloc(ha.size());
    cg.alloc(hc.size());
    kd.alloc(hk.size());
    s.alloc(ha.size());
    d.alloc(ha.size());
    WWB_CHECK(cudaMemcpy(a.ptr, ha.data(), ha.size() * 4, cudaMemcpyHostToDevice));
    WWB_CHECK(cudaMemcpy(cg.ptr, hc.data(), hc.size() * 4, cudaMemcpyHostToDevice));
    WWB_CHECK(cudaMemcpy(kd.ptr, hk.data(), hk.size() * 4, cudaMemcpyHostToDevice));
    cudaStream_t st = runtime().stream;
    const std::string key = "dia " + std::to_string(c.cfg.nk) + "x" + std::to_string(c.cfg.nth) +
                            " " + tune::device_key();
    const int k = tune::pick(
        key, cands,
        [&](int kern, cudaStream_t ss) {
          launch_snl1(kern, c.dev, n, a.ptr, cg.ptr, kd.ptr, s.ptr, d.ptr, ss);
        },
        nullptr, st, 3);
    WWB_CHECK(cudaStreamSynchronize(st));
    c.kernel = k;
    g_status.ok();
    return k;
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
    return -1;
  }
}

int ww_snl1_select_kernel(int igrid, int which) {
  auto it = contexts().find(igrid);
  if (it == contexts().end() || !it->second->ready) return -1;
  Ctx& c = *it->second;
  const int k = pick_kernel(c, which);
  if (k < 0) return -1;
  const int prev = c.kernel;
  c.kernel = k;
  return prev;
}

}  // extern "C"
