// ww3-gpu_b200/csrc/abi_st4.cpp
// The ST4 part of the C ABI: ww_st4_init / set_real / set_int / commit (the grid's scalars and
// arrays, copied to the device at commit), the point entries ww_sds4 / ww_sin4 / ww_spr4 on host
// arrays, ww_st4_enabled, ww_st4_last_error, and the state W3SRCE reads (st4_grid_dev).
//
// Reference: ww3-gpu kokkos/src/fortran_iface/st4_shim.cpp:472-760 and ww_kokkos_c.hpp:136-203:
// status codes (NOT_INITIALISED before init, BAD_SHAPE for packet lengths, UNSUPPORTED for
// W3_FLX5, TABLE for a bad registration or a missing / short array at commit), module arrays one
// per process with the last registration winning, OUT arguments copied in as well as out,
// npts == 0 a no-op. WW_KOKKOS_ST4_TABLES=1 makes ww_st4_commit rebuild the tables with INSIN4
// (the reference: its C++ on the host, st4_shim.cpp:301-345; here: st4_tables_kernel.cu on the
// device), print how many values differ from the registered ones and use the rebuilt ones.
// ww_st4_tables runs the same device INSIN4 on a packet and host arrays and returns its tables.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "st4_registry.hpp"
#include "st4_srce.cuh"
#include "st4_tables_kernel.cuh"
#include "staging.hpp"
#include "step.hpp"
#include "wwb_common.hpp"

namespace wwb {
namespace {

Status g_status;

/// A device copy of a host vector, owned.
template <class T>
struct DevVec {
  T* ptr = nullptr;
  size_t n = 0;
  DevVec() = default;
  DevVec(const DevVec&) = delete;
  DevVec& operator=(const DevVec&) = delete;
  ~DevVec() { free_table(ptr); }
  void upload(const std::vector<T>& h) {
    free_table(ptr);
    ptr = nullptr;
    n = h.size();
    if (n == 0) return;
    WWB_CHECK(cudaMalloc(&ptr, n * sizeof(T)));
    WWB_CHECK(cudaMemcpy(ptr, h.data(), n * sizeof(T), cudaMemcpyHostToDevice));
  }
};

/// A grid: its registrations, and after commit its device arrays and kernel parameters.
struct GridCtx {
  st4::GridReg reg;
  bool ready = false;
  DevVec<float> f[st4::NARRAYS];
  DevVec<int> i[st4::NARRAYS];
  DevVec<float> satw_t;
  DevVec<int> sati_t;
  DevVec<float> cumulw_t;
  St4Dev host{};                    ///< the kernel parameters (module state of the commit)
  St4Dev* dev = nullptr;            ///< their device copy
  ~GridCtx() {
    if (dev) cudaFree(dev);
  }
};

struct ModuleCtx {
  st4::ModuleReg reg;
  DevVec<float> f[st4::NARRAYS];
};

std::map<int, std::unique_ptr<GridCtx>>& grids() {
  static auto* m = new std::map<int, std::unique_ptr<GridCtx>>();
  return *m;
}
ModuleCtx& module_ctx() {
  static auto* m = new ModuleCtx();
  return *m;
}

/// The kernel parameters of grid g with the module's current arrays and DEL* scalars, copied to
/// g's device struct (the reference reads the module state at every call).
void refresh(GridCtx& g) {
  ModuleCtx& m = module_ctx();
  const auto& a = g.reg.a;
  st4::FieldPtrs q{g.f[st4::A_SIG].ptr,   g.f[st4::A_SIG2].ptr,  g.f[st4::A_DSIP].ptr,
                   g.f[st4::A_DDEN].ptr,  g.f[st4::A_DDEN2].ptr, g.f[st4::A_ESIN].ptr,
                   g.f[st4::A_ECOS].ptr,  g.f[st4::A_TH].ptr,    g.satw_t.ptr,
                   g.cumulw_t.ptr, g.f[st4::A_DCKI].ptr, g.f[st4::A_QBI].ptr,
                   m.f[st4::A_TAUT].ptr,  m.f[st4::A_TAUHFT].ptr, m.f[st4::A_TAUHFT2].ptr,
                   m.f[st4::A_FWTABLE].ptr, g.sati_t.ptr,         g.i[st4::A_IKTAB].ptr};
  (void)a;
  g.host.p = st4::current_params(g.reg, m.reg);
  g.host.f = st4::make_fields(g.reg, q);
  if (g.dev == nullptr) WWB_CHECK(cudaMalloc(&g.dev, sizeof(St4Dev)));
  WWB_CHECK(cudaMemcpy(g.dev, &g.host, sizeof(St4Dev), cudaMemcpyHostToDevice));
}

GridCtx* compute_ctx(int igrid, int npts, const char* who) {
  auto it = grids().find(igrid);
  if (it == grids().end() || !it->second->ready || !runtime().ready) {
    g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED,
                  (std::string(who) + " before ww_st4_commit for this grid").c_str());
    return nullptr;
  }
  if (npts < 0) {
    g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, (std::string(who) + ": npts < 0").c_str());
    return nullptr;
  }
  if (npts == 0) {
    g_status.ok();
    return nullptr;
  }
  return it->second.get();
}

/// Staging slots taken in call order: reset() at the start of a call, then one in() per array.
struct Cursor {
  Staging st;
  size_t next = 0;
  void reset() { next = 0; }
  template <class T>
  T* in(const T* h, size_t n, cudaStream_t s) {
    return st.in(next++, h, n, s);
  }
  void release() { st.release(); }
};

Cursor& staging() {
  static auto* s = new Cursor();
  return *s;
}

/// Copies a host array of n floats or ints into the device staging area; returns the pointer.
template <class T>
T* in(const T* h, size_t n, cudaStream_t s) {
  return staging().in(h, n, s);
}

template <class T>
void out(T* h, const T* d, size_t n, cudaStream_t s) {
  if (n) WWB_CHECK(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
}


/// INSIN4's tables on the host, as the device builds them (shapes of st4_tables_kernel.cuh).
struct HostTables {
  std::vector<float> satweights, dcki, qbi, cumulw, taut, tauhft, tauhft2;
  std::vector<int> satindices, iktab;
};

/// A device buffer of n elements, freed on scope exit.
template <class T>
struct Scratch {
  T* ptr = nullptr;
  explicit Scratch(size_t n) {
    if (n) WWB_CHECK(cudaMalloc(&ptr, n * sizeof(T)));
  }
  ~Scratch() {
    if (ptr) cudaFree(ptr);
  }
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
};

/// Runs INSIN4(FLTABS) on the device for packet p with SIG, DSIP (0:MK+1), TH (MTH), ECOS
/// (MSPEC+MTH) from the host and brings every table back; the TABU_* tables only where INSIN4
/// builds them. Returns INSIN4's branches and DEL* values.
St4TablesPlan build_tables(const st4::Params& p, bool fltabs, const float* sig, const float* dsip,
                           const float* th, const float* ecos, HostTables& t) {
  const St4TablesPlan q = st4_tables_plan(p, fltabs);
  cudaStream_t s = runtime().stream;
  cudaStream_t s2 = nullptr;
  WWB_CHECK(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t st;
    ~StreamGuard() { cudaStreamDestroy(st); }
  } guard{s2};
  const size_t nsig = static_cast<size_t>(p.mk) + 2;
  Scratch<float> d_sig(nsig), d_dsip(nsig), d_th(p.mth), d_ecos(p.mspec + p.mth);
  WWB_CHECK(cudaMemcpyAsync(d_sig.ptr, sig, nsig * 4, cudaMemcpyHostToDevice, s));
  WWB_CHECK(cudaMemcpyAsync(d_dsip.ptr, dsip, nsig * 4, cudaMemcpyHostToDevice, s));
  WWB_CHECK(cudaMemcpyAsync(d_th.ptr, th, sizeof(float) * p.mth, cudaMemcpyHostToDevice, s));
  WWB_CHECK(cudaMemcpyAsync(d_ecos.ptr, ecos, sizeof(float) * (p.mspec + p.mth),
                            cudaMemcpyHostToDevice, s));
  const size_t nsat = static_cast<size_t>(q.nsat) * p.mth, nik = static_cast<size_t>(p.mk) * st4::kNdtab;
  const size_t ntab = static_cast<size_t>(st4::kNkhs) * st4::kNkd;
  const size_t ncum = static_cast<size_t>(p.mspec) * p.mspec;
  const size_t ntaut = (q.taut ? static_cast<size_t>(st4::kItauMax + 1) * (st4::kJuMax + 1) : 0);
  const size_t nhf = (q.tauhf || q.tauhf2)
                         ? static_cast<size_t>(st4::kIustar + 1) * (st4::kIalpha + 1) : 0;
  const size_t nhf2 = q.tauhf2 ? nhf * (st4::kIlevTail + 1) : 0;
  Scratch<float> satw(nsat), dcki(ntab), qbi(ntab), cumulw(ncum), taut(ntaut), tauhft(nhf),
      tauhft2(nhf2);
  Scratch<int> sati(nsat), iktab(nik);
  St4TablesOut o{satw.ptr, sati.ptr, iktab.ptr, dcki.ptr, qbi.ptr, cumulw.ptr,
                 taut.ptr, tauhft.ptr, tauhft2.ptr};
  launch_st4_tables(p, q, St4TablesIn{d_sig.ptr, d_dsip.ptr, d_th.ptr, d_ecos.ptr}, o, s, s2);
  auto back = [&](auto& v, const auto* d, size_t n) {
    v.resize(n);
    if (n) WWB_CHECK(cudaMemcpyAsync(v.data(), d, n * sizeof(v[0]), cudaMemcpyDeviceToHost, s));
  };
  back(t.satweights, satw.ptr, nsat);
  back(t.satindices, sati.ptr, nsat);
  back(t.iktab, iktab.ptr, nik);
  back(t.dcki, dcki.ptr, ntab);
  back(t.qbi, qbi.ptr, ntab);
  back(t.cumulw, cumulw.ptr, ncum);
  back(t.taut, taut.ptr, ntaut);
  back(t.tauhft, tauhft.ptr, nhf);
  back(t.tauhft2, tauhft2.ptr, nhf2);
  WWB_CHECK(cudaStreamSynchronize(s));
  return q;
}

/// Values of b that are not bitwise equal to a's (a missing array counts all of b).
template <class T>
long long count_diff(const std::vector<T>& a, const std::vector<T>& b) {
  if (a.size() != b.size()) return static_cast<long long>(b.size());
  long long n = 0;
  for (size_t k = 0; k < a.size(); ++k)
    if (std::memcmp(&a[k], &b[k], sizeof(T)) != 0) ++n;
  return n;
}

/// WW_KOKKOS_ST4_TABLES=1 at commit: grid g's and the module's tables rebuilt by the device
/// INSIN4(FLTABS=.TRUE.) from g's registered SIG, DSIP, TH and ECOS; the count of values that
/// differ from the registered ones is printed, and the rebuilt ones replace them. TAUT/TAUHFT
/// (SINTAILPAR(1) > 0.5) and TAUHFT2 (also TTAUWSHELTER > 0) and their DEL* change only where
/// INSIN4 builds them, as the Fortran's module state does.
void rebuild_tables(GridCtx& g, ModuleCtx& m) {
  const st4::Params& p = g.reg.p;
  HostTables t;
  const St4TablesPlan q = build_tables(p, true, g.reg.a[st4::A_SIG].f.data(),
                                       g.reg.a[st4::A_DSIP].f.data(),
                                       g.reg.a[st4::A_TH].f.data(),
                                       g.reg.a[st4::A_ECOS].f.data(), t);
  auto& ga = g.reg.a;
  auto& ma = m.reg.a;
  long long diff = count_diff(ga[st4::A_SATWEIGHTS].f, t.satweights) +
                   count_diff(ga[st4::A_SATINDICES].i, t.satindices) +
                   count_diff(ga[st4::A_IKTAB].i, t.iktab) + count_diff(ga[st4::A_DCKI].f, t.dcki) +
                   count_diff(ga[st4::A_QBI].f, t.qbi) + count_diff(ga[st4::A_CUMULW].f, t.cumulw);
  if (q.taut) diff += count_diff(ma[st4::A_TAUT].f, t.taut);
  if (q.tauhf || q.tauhf2) diff += count_diff(ma[st4::A_TAUHFT].f, t.tauhft);
  if (q.tauhf2) diff += count_diff(ma[st4::A_TAUHFT2].f, t.tauhft2);
  std::fprintf(stderr,
               "ww_b200: ST4 tables rebuilt on the device: %lld values differ from the "
               "registered ones\n",
               diff);
  ga[st4::A_SATWEIGHTS].f = std::move(t.satweights);
  ga[st4::A_SATINDICES].i = std::move(t.satindices);
  ga[st4::A_IKTAB].i = std::move(t.iktab);
  ga[st4::A_DCKI].f = std::move(t.dcki);
  ga[st4::A_QBI].f = std::move(t.qbi);
  ga[st4::A_CUMULW].f = std::move(t.cumulw);
  if (q.taut) {
    ma[st4::A_TAUT].f = std::move(t.taut);
    m.reg.delu = q.delu;
    m.reg.deltauw = q.deltauw;
  }
  if (q.tauhf || q.tauhf2) {
    ma[st4::A_TAUHFT].f = std::move(t.tauhft);
    m.reg.delust = q.delust;
    m.reg.delalp = q.delalp;
  }
  if (q.tauhf2) {
    ma[st4::A_TAUHFT2].f = std::move(t.tauhft2);
    m.reg.deltail = q.deltail;
  }
}

}  // namespace

/// The committed ST4 state of grid igrid for W3SRCE: scalars, fields (device pointers).
bool st4_grid_dev(int igrid, St4Dev* out_state) {
  auto it = grids().find(igrid);
  if (it == grids().end() || !it->second->ready) return false;
  refresh(*it->second);
  *out_state = it->second->host;
  return true;
}

void release_st4_contexts() {
  grids().clear();
  ModuleCtx& m = module_ctx();
  for (auto& v : m.f) v.upload({});
  staging().release();
}

}  // namespace wwb

using namespace wwb;

extern "C" {

int ww_st4_init(int igrid, const float* rpar, int nrpar, const int* ipar, int nipar) {
  try {
    grids().erase(igrid);
    if (!runtime().ready)
      return g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_st4_init before ww_kokkos_init");
    if (rpar == nullptr || ipar == nullptr || nrpar != st4::NRPAR || nipar != st4::NIPAR)
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                           "ww_st4_init: RPAR/IPAR length differs from the ST4 packet layout");
    if (ipar[st4::I_FLX5] != 0)
      return g_status.fail(WW_KOKKOS_ERR_UNSUPPORTED, "ww_st4_init: W3_FLX5 is not supported");
    const st4::Params p = st4::unpack(rpar, ipar);
    if (p.nk <= 0 || p.nth <= 0 || p.nspec != p.nk * p.nth || p.mk < p.nk || p.mth < p.nth ||
        p.mspec < p.nspec)
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                           "ww_st4_init: NK, NTH, NSPEC, MK, MTH, MSPEC inconsistent");
    if (p.nth > 128)
      return g_status.fail(WW_KOKKOS_ERR_UNSUPPORTED, "ww_st4_init: more than 128 directions");
    auto g = std::make_unique<GridCtx>();
    g->reg.p = p;
    g->reg.configured = true;
    st4::ModuleReg& m = module_ctx().reg;  // module scalars: the last grid to initialise wins
    m.delust = p.delust;
    m.delalp = p.delalp;
    m.deltauw = p.deltauw;
    m.delu = p.delu;
    m.deltail = p.deltail;
    m.delab = p.delab;
    grids()[igrid] = std::move(g);
    g_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    grids().erase(igrid);
    return g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  }
}

static int set_array(int igrid, int id, const void* data, bool is_int, int rank,
                     const int* lbound, const int* extent) {
  auto it = grids().find(igrid);
  if (it == grids().end() || !it->second->reg.configured)
    return g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED,
                         "ww_st4_set_* before ww_st4_init for this grid");
  std::string why;
  const int rc = st4::reg_set(it->second->reg, module_ctx().reg, id, data, is_int, rank, lbound,
                              extent, why);
  if (rc != 0) return g_status.fail(rc, ("ww_st4_set_*: " + why).c_str());
  it->second->ready = false;
  g_status.ok();
  return WW_KOKKOS_OK;
}

int ww_st4_set_real(int igrid, int id, const float* data, int rank, const int* lbound,
                    const int* extent) {
  try {
    return set_array(igrid, id, data, false, rank, lbound, extent);
  } catch (const std::exception& e) {
    return g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  }
}

int ww_st4_set_int(int igrid, int id, const int* data, int rank, const int* lbound,
                   const int* extent) {
  try {
    return set_array(igrid, id, data, true, rank, lbound, extent);
  } catch (const std::exception& e) {
    return g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  }
}

int ww_st4_tables(const float* rpar, int nrpar, const int* ipar, int nipar, const float* sig,
                  const float* dsip, const float* th, const float* ecos, int fltabs,
                  float* satweights, int* satindices, int* iktab, float* dcki, float* qbi,
                  float* cumulw, float* taut, float* tauhft, float* tauhft2, float* del) {
  try {
    if (!runtime().ready)
      return g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_st4_tables before ww_kokkos_init");
    if (rpar == nullptr || ipar == nullptr || nrpar != st4::NRPAR || nipar != st4::NIPAR ||
        !sig || !dsip || !th || !ecos || !del)
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_st4_tables: bad packet or null array");
    const st4::Params p = st4::unpack(rpar, ipar);
    if (p.nk <= 0 || p.nth <= 1 || p.nspec != p.nk * p.nth || p.mk < p.nk || p.mth < p.nth ||
        p.mspec < p.nspec)
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                           "ww_st4_tables: NK, NTH, NSPEC, MK, MTH, MSPEC inconsistent");
    HostTables t;
    const St4TablesPlan q = build_tables(p, fltabs != 0, sig, dsip, th, ecos, t);
    auto put = [](auto* dst, const auto& v) {
      if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    put(satweights, t.satweights);
    put(satindices, t.satindices);
    put(iktab, t.iktab);
    put(dcki, t.dcki);
    put(qbi, t.qbi);
    put(cumulw, t.cumulw);
    put(taut, t.taut);
    put(tauhft, t.tauhft);
    put(tauhft2, t.tauhft2);
    del[0] = q.delust;
    del[1] = q.delalp;
    del[2] = q.deltauw;
    del[3] = q.delu;
    del[4] = q.deltail;
    g_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::bad_alloc& e) {
    return g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  } catch (const std::exception& e) {
    return g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_st4_commit(int igrid) {
  try {
    auto it = grids().find(igrid);
    if (it == grids().end() || !it->second->reg.configured || !runtime().ready)
      return g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED,
                           "ww_st4_commit before ww_st4_init for this grid");
    GridCtx& g = *it->second;
    ModuleCtx& m = module_ctx();
    std::string why;
    if (!st4::reg_check(g.reg, m.reg, why))
      return g_status.fail(WW_KOKKOS_ERR_TABLE, ("ww_st4_commit: " + why).c_str());
    if (ww_kokkos_flag("WW_KOKKOS_ST4_TABLES") != 0) rebuild_tables(g, m);
    for (int id = 0; id < st4::NARRAYS; ++id) {
      if (st4::kArraySpecs[id].module) {
        m.f[id].upload(m.reg.a[id].f);
      } else if (st4::kArraySpecs[id].is_int) {
        g.i[id].upload(g.reg.a[id].i);
      } else {
        g.f[id].upload(g.reg.a[id].f);
      }
    }
    std::vector<float> wt;
    std::vector<int> itt;
    st4::transpose_sat(g.reg, wt, itt);
    g.satw_t.upload(wt);
    g.sati_t.upload(itt);
    std::vector<float> ct;
    st4::transpose_cumulw(g.reg, ct);
    g.cumulw_t.upload(ct);
    g.f[st4::A_CUMULW].upload({});  // only the transposed copy is read
    refresh(g);
    g.ready = true;
    g_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::bad_alloc& e) {
    return g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  } catch (const std::exception& e) {
    return g_status.fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  }
}

void ww_sds4(int igrid, int npts, const float* a, const float* k, const float* cg,
             const float* ustar, const float* usdir, const float* depth, const float* dair,
             const float* dlwmean, int flogrd57, int flogrd58, float* srhs, float* ddiag,
             float* brlambda, float* whitecap) {
  try {
    GridCtx* g = compute_ctx(igrid, npts, "ww_sds4");
    if (g == nullptr) return;
    if (!a || !k || !cg || !ustar || !usdir || !depth || !dair || !dlwmean || !srhs || !ddiag ||
        !brlambda || !whitecap) {
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sds4: null array");
      return;
    }
    refresh(*g);
    const size_t n = npts, ns = n * g->host.p.nspec, nk = n * g->host.p.nk;
    cudaStream_t s = runtime().stream;
    staging().reset();
    const float *da = in(a, ns, s), *dk = in(k, nk, s), *dcg = in(cg, nk, s);
    const float *du = in(ustar, n, s), *dd = in(usdir, n, s), *ddep = in(depth, n, s);
    const float *dair_ = in(dair, n, s), *dlw = in(dlwmean, n, s);
    float *ds = in(srhs, ns, s), *ddg = in(ddiag, ns, s), *db = in(brlambda, ns, s);
    float* dwc = in(whitecap, 4 * n, s);
    launch_sds4(g->dev, g->host.p, npts, da, dk, dcg, du, dd, ddep, dair_, dlw, flogrd57, flogrd58,
                ds, ddg, db, dwc, s);
    out(srhs, ds, ns, s);
    out(ddiag, ddg, ns, s);
    out(brlambda, db, ns, s);
    out(whitecap, dwc, 4 * n, s);
    WWB_CHECK(cudaStreamSynchronize(s));
    g_status.ok();
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

void ww_sin4(int igrid, int npts, const float* a, const float* cg, const float* k, const float* u,
             const float* ustar, const float* drat, const float* as, const float* usdir,
             const float* z0, const float* cd, float* tauwx, float* tauwy, float* tauwnx,
             float* tauwny, float* s, float* d, int* llws) {
  try {
    GridCtx* g = compute_ctx(igrid, npts, "ww_sin4");
    if (g == nullptr) return;
    if (!a || !cg || !k || !u || !ustar || !drat || !as || !usdir || !z0 || !cd || !tauwx ||
        !tauwy || !tauwnx || !tauwny || !s || !d || !llws) {
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_sin4: null array");
      return;
    }
    refresh(*g);
    const size_t n = npts, ns = n * g->host.p.nspec, nk = n * g->host.p.nk;
    cudaStream_t st = runtime().stream;
    staging().reset();
    const float *da = in(a, ns, st), *dcg = in(cg, nk, st), *dk = in(k, ns, st);
    const float *du = in(u, n, st), *dus = in(ustar, n, st), *ddr = in(drat, n, st);
    const float *das = in(as, n, st), *dud = in(usdir, n, st), *dz0 = in(z0, n, st);
    float *tx = in(tauwx, n, st), *ty = in(tauwy, n, st), *tnx = in(tauwnx, n, st),
          *tny = in(tauwny, n, st);
    float *ds = in(s, ns, st), *dd = in(d, ns, st);
    int* dl = in(llws, ns, st);
    launch_sin4(g->dev, g->host.p, npts, da, dcg, dk, du, dus, ddr, das, dud, dz0, tx, ty, tnx,
                tny, ds, dd, dl, st);
    out(tauwx, tx, n, st);
    out(tauwy, ty, n, st);
    out(tauwnx, tnx, n, st);
    out(tauwny, tny, n, st);
    out(s, ds, ns, st);
    out(d, dd, ns, st);
    out(llws, dl, ns, st);
    WWB_CHECK(cudaStreamSynchronize(st));
    g_status.ok();
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

void ww_spr4(int igrid, int npts, const float* a, const float* cg, const float* wn,
             const float* u, const float* udir, const float* tauwx, const float* tauwy,
             const int* llws, float* ustar, float* usdir, float* emean, float* fmean,
             float* fmean1, float* wnmean, float* amax, float* cd, float* z0, float* charn,
             float* fmeanws, float* dlwmean) {
  try {
    GridCtx* g = compute_ctx(igrid, npts, "ww_spr4");
    if (g == nullptr) return;
    float* host12[12] = {ustar, usdir, emean, fmean, fmean1, wnmean,
                         amax,  cd,    z0,    charn, fmeanws, dlwmean};
    bool null = !a || !cg || !wn || !u || !udir || !tauwx || !tauwy || !llws;
    for (float* h : host12) null = null || h == nullptr;
    if (null) {
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_spr4: null array");
      return;
    }
    refresh(*g);
    const size_t n = npts, ns = n * g->host.p.nspec, nk = n * g->host.p.nk;
    cudaStream_t st = runtime().stream;
    staging().reset();
    const float *da = in(a, ns, st), *dcg = in(cg, nk, st), *dwn = in(wn, nk, st);
    const float *du = in(u, n, st), *dud = in(udir, n, st), *dtx = in(tauwx, n, st),
                *dty = in(tauwy, n, st);
    const int* dl = in(llws, ns, st);
    float* dev12[12];
    for (int j = 0; j < 12; ++j) dev12[j] = in(host12[j], n, st);
    launch_spr4(g->dev, g->host.p, npts, da, dcg, dwn, du, dud, dtx, dty, dl, dev12, st);
    for (int j = 0; j < 12; ++j) out(host12[j], dev12[j], n, st);
    WWB_CHECK(cudaStreamSynchronize(st));
    g_status.ok();
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_st4_enabled(int which) {
  static const char* names[] = {"", "WW_KOKKOS_SDS4", "WW_KOKKOS_SIN4", "WW_KOKKOS_SPR4",
                                "WW_KOKKOS_ST4_TABLES"};
  if (which < 1 || which > 4) return 0;
  return ww_kokkos_flag(names[which]) != 0 ? 1 : 0;
}

int ww_st4_last_error(void) { return g_status.get(); }

}  // extern "C"
