// ww3-gpu_b200/csrc/abi_srce.cpp
// The W3SRCE part of the C ABI: ww_srce_init, ww_srce (one point), ww_srce_batch (the points of a
// time step, host arrays), ww_srce_batch_va (the same on the resident VA), ww_srce_enabled,
// ww_srce_last_error.
//
// Reference: ww3-gpu kokkos/src/fortran_iface/srce_shim.cpp:679-1046 and ww_kokkos_c.hpp:205-276,
// resident_c.hpp:86-101: ww_srce_init needs ww_snl1_init and ww_st4_commit of the same grid
// (NOT_INITIALISED otherwise), refuses packets of another length (BAD_SHAPE) and builds other
// than switch_lab_shrd's source terms (UNSUPPORTED); every call reads the DIA and ST4 state of the
// grid as it is then; the batch entries take every per-point array packed point by point
// (Fortran (rows, npts)); npts == 0 is a no-op. W3FLD2 (I_FLD2) is not built here and is refused
// as UNSUPPORTED, as are DIA tables that are not in the row-shift form.
#include <cuda_runtime.h>

#include <algorithm>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "autotune.hpp"
#include "st4_srce.cuh"
#include "staging.hpp"
#include "step.hpp"
#include "va.hpp"
#include "wwb_common.hpp"

namespace wwb {

bool snl1_grid_dev(int igrid, Snl1Dev* out);   // abi_snl1.cpp
bool st4_grid_dev(int igrid, St4Dev* out);      // abi_st4.cpp

namespace {

Status g_status;

template <class T>
struct DevVec {
  T* ptr = nullptr;
  DevVec() = default;
  DevVec(const DevVec&) = delete;
  DevVec& operator=(const DevVec&) = delete;
  ~DevVec() { free_table(ptr); }
  void upload(const T* h, size_t n) {
    free_table(ptr);
    ptr = nullptr;
    WWB_CHECK(cudaMalloc(&ptr, (n ? n : 1) * sizeof(T)));
    if (n) WWB_CHECK(cudaMemcpy(ptr, h, n * sizeof(T), cudaMemcpyHostToDevice));
  }
};

struct GridCtx {
  srce::Params p{};
  DevVec<float> sig, dden, ecos, esin;
  DevVec<int> mapwn;
  SrceDev* dev = nullptr;   ///< device copy of the launch parameters, rebuilt at every call
  SrceWork work;            ///< the work queue's counter, the working sets' global part
  ~GridCtx() {
    if (dev) cudaFree(dev);
    work.release();
  }
};

std::map<int, std::unique_ptr<GridCtx>>& grids() {
  static auto* m = new std::map<int, std::unique_ptr<GridCtx>>();
  return *m;
}

struct Cursor {
  Staging st;
  size_t next = 0;
  template <class T>
  T* in(const T* h, size_t n, cudaStream_t s) {
    return st.in(next++, h, n, s);
  }
};
Cursor& staging() {
  static auto* s = new Cursor();
  return *s;
}

template <class T>
void out(T* h, const T* d, size_t n, cudaStream_t s) {
  if (n) WWB_CHECK(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
}

/// The launch parameters of grid g from the DIA and ST4 state of igrid now; false (status set)
/// when either is gone.
bool prepare(int igrid, GridCtx& g, SrceDev& host, const char* who) {
  Snl1Dev n{};
  St4Dev q{};
  if (!snl1_grid_dev(igrid, &n) || !st4_grid_dev(igrid, &q)) {
    g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED,
                  (std::string(who) + ": the DIA or ST4 context of this grid is gone").c_str());
    return false;
  }
  host.p = g.p;
  host.g = pt::SrceGrid{g.sig.ptr, g.dden.ptr, g.ecos.ptr, g.esin.ptr, g.mapwn.ptr};
  host.q = q.p;
  host.f = q.f;
  host.n = n;
  host.L = pt::srce_layout(q.p, n);
  if (g.dev == nullptr) WWB_CHECK(cudaMalloc(&g.dev, sizeof(SrceDev)));
  WWB_CHECK(cudaMemcpy(g.dev, &host, sizeof(SrceDev), cudaMemcpyHostToDevice));
  return true;
}

/// The batch on host arrays (spec_dev null) or on the resident VA (spec_dev, jsea_host).
void run_batch(int igrid, GridCtx& g, const SrceStep& step, int npts, float* spec, float* va_dev,
               const int* jsea, const float* wn1, const float* cg1, const float* pin, float* psc,
               float* whitecap, float* taubbl, float* tauice, int* shave, const char* who) {
  SrceDev host{};
  if (!prepare(igrid, g, host, who)) return;
  const size_t n = npts, ns = n * g.p.nspec, nk = n * g.p.nk;
  if (StepRecorder* rec = va_dev ? step_recorder(igrid) : nullptr) {
    // A recorded step: the launch parameters, the inputs and the work buffers are the step's
    // own; the per-point packets (PSC, WHITECAP, TAUBBL, TAUICE, SHAVE) stay on the device and
    // carry over from one replay to the next.
    cudaStream_t s = step_stream(rec);
    auto cur = std::make_shared<Cursor>();
    auto work = std::shared_ptr<SrceWork>(new SrceWork(), [](SrceWork* w) {
      w->release();
      delete w;
    });
    SrceDev* d = nullptr;
    WWB_CHECK(cudaMalloc(&d, sizeof(SrceDev)));
    auto dk = std::shared_ptr<SrceDev>(d, [](SrceDev* p) { cudaFree(p); });
    WWB_CHECK(cudaMemcpy(d, &host, sizeof(SrceDev), cudaMemcpyHostToDevice));
    const int* djsea = cur->in(jsea, n, s);
    const float *dwn = cur->in(wn1, nk, s), *dcg = cur->in(cg1, nk, s),
                *dpin = cur->in(pin, n * srce::NPIN, s);
    float* dpsc = cur->in(psc, n * srce::NPSC, s);
    float *dwc = cur->in(whitecap, 4 * n, s), *dtb = cur->in(taubbl, 2 * n, s),
          *dti = cur->in(tauice, 2 * n, s);
    int* dsh = cur->in(shave, n, s);
    srce_reserve(host.L, npts, *work, s);
    WWB_CHECK(cudaStreamSynchronize(s));
    step_keep(rec, cur);
    step_keep(rec, work);
    step_keep(rec, dk);
    const pt::SrceLayout L = host.L;
    SrceWork* const w = work.get();
    auto job = std::make_shared<SrceRecorded>();
    job->job = SrceJob{d, step, npts, 0, va_dev, djsea, dwn, dcg, dpin, dpsc, dwc, dtb, dti, dsh};
    job->L = L;
    step_add(
        rec,
        [=](cudaStream_t ss) {
          launch_srce(d, L, step, npts, va_dev, djsea, dwn, dcg, dpin, dpsc, dwc, dtb, dti, dsh,
                      *w, ss);
        },
        job);
    g_status.ok();
    return;
  }
  cudaStream_t s = runtime().stream;
  Cursor& c = staging();
  c.next = 0;
  float* dspec = va_dev ? va_dev : c.in(spec, ns, s);
  const int* djsea = jsea ? c.in(jsea, n, s) : nullptr;
  const float *dwn = c.in(wn1, nk, s), *dcg = c.in(cg1, nk, s),
              *dpin = c.in(pin, n * srce::NPIN, s);
  float* dpsc = c.in(psc, n * srce::NPSC, s);
  float *dwc = c.in(whitecap, 4 * n, s), *dtb = c.in(taubbl, 2 * n, s),
        *dti = c.in(tauice, 2 * n, s);
  int* dsh = c.in(shave, n, s);
  launch_srce(g.dev, host.L, step, npts, dspec, djsea, dwn, dcg, dpin, dpsc, dwc, dtb, dti, dsh,
              g.work, s);
  if (!va_dev) out(spec, dspec, ns, s);
  out(psc, dpsc, n * srce::NPSC, s);
  out(whitecap, dwc, 4 * n, s);
  out(taubbl, dtb, 2 * n, s);
  out(tauice, dti, 2 * n, s);
  out(shave, dsh, n, s);
  WWB_CHECK(cudaStreamSynchronize(s));
  g_status.ok();
}

GridCtx* find(int igrid, const char* who) {
  auto it = grids().find(igrid);
  if (it == grids().end() || !runtime().ready) {
    g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED,
                  (std::string(who) + " before ww_srce_init for this grid").c_str());
    return nullptr;
  }
  return it->second.get();
}

}  // namespace

void release_srce_contexts() {
  grids().clear();
  staging().st.release();
}

}  // namespace wwb

using namespace wwb;

extern "C" {

int ww_srce_init(int igrid, const float* rpar, int nrpar, const int* ipar, int nipar,
                 const float* sig, const float* dden, const float* ecos, const float* esin,
                 const int* mapwn) {
  try {
    grids().erase(igrid);
    if (!runtime().ready)
      return g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_srce_init before ww_kokkos_init");
    if (nrpar != srce::NRPAR || nipar != srce::NIPAR || !rpar || !ipar || !sig || !dden ||
        !ecos || !esin || !mapwn)
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                           "ww_srce_init: RPAR/IPAR length differs from the W3SRCE packet layout");
    if (ipar[srce::I_LAB_SWITCH] != 1)
      return g_status.fail(WW_KOKKOS_ERR_UNSUPPORTED,
                           "ww_srce_init: only switch_lab_shrd's source terms are translated");
    const srce::Params p = srce::unpack(rpar, ipar);
    if (p.nk <= 0 || p.nth <= 0 || p.nspec != p.nk * p.nth)
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_srce_init: nspec != nk*nth");
    Snl1Dev n{};
    St4Dev q{};
    if (!snl1_grid_dev(igrid, &n) || !st4_grid_dev(igrid, &q))
      return g_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED,
                           "ww_srce_init before ww_snl1_init and ww_st4_commit for this grid");
    if (n.nk != p.nk || n.nth != p.nth || q.p.nk != p.nk || q.p.nth != p.nth)
      return g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                           "ww_srce_init: NK/NTH differ from the DIA or ST4 context");
    if (p.fld2 != 0)
      return g_status.fail(WW_KOKKOS_ERR_UNSUPPORTED, "ww_srce_init: W3FLD2 is not built");
    if (srce_smem_bytes(pt::srce_layout(q.p, n)) == 0)
      return g_status.fail(WW_KOKKOS_ERR_UNSUPPORTED,
                           "ww_srce_init: the point's working set exceeds a CTA's shared memory");
    auto g = std::make_unique<GridCtx>();
    g->p = p;
    g->sig.upload(sig, p.nk);
    g->dden.upload(dden, p.nk);
    g->ecos.upload(ecos, p.nspec);
    g->esin.upload(esin, p.nspec);
    g->mapwn.upload(mapwn, p.nspec);
    grids()[igrid] = std::move(g);
    g_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    grids().erase(igrid);
    return g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

void ww_srce_batch(int igrid, int it, int inflags24, int flogrd57, int flogrd58, float dtg,
                   int npts, float* spec, const float* wn1, const float* cg1, const float* pin,
                   float* psc, float* whitecap, float* taubbl, float* tauice, int* shave) {
  try {
    GridCtx* g = find(igrid, "ww_srce_batch");
    if (g == nullptr) return;
    if (npts < 0 || (npts > 0 && (!spec || !wn1 || !cg1 || !pin || !psc || !whitecap ||
                                  !taubbl || !tauice || !shave))) {
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_srce_batch: npts < 0 or a null array");
      return;
    }
    if (npts == 0) {
      g_status.ok();
      return;
    }
    timers::Region t("srce.batch.call");
    run_batch(igrid, *g, SrceStep{it, inflags24, flogrd57, flogrd58, dtg}, npts, spec, nullptr,
              nullptr, wn1, cg1, pin, psc, whitecap, taubbl, tauice, shave, "ww_srce_batch");
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

void ww_srce_batch_va(int igrid, int it, int inflags24, int flogrd57, int flogrd58, float dtg,
                      float* va, int nspec, int nsealm, int npts, const int* jsea,
                      const float* wn1, const float* cg1, const float* pin, float* psc,
                      float* whitecap, float* taubbl, float* tauice, int* shave) {
  try {
    GridCtx* g = find(igrid, "ww_srce_batch_va");
    if (g == nullptr) return;
    if (npts < 0 || (npts > 0 && (!va || !jsea || !wn1 || !cg1 || !pin || !psc || !whitecap ||
                                  !taubbl || !tauice || !shave))) {
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_srce_batch_va: npts < 0 or a null array");
      return;
    }
    if (nspec != g->p.nspec || npts > nsealm) {
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE,
                    "ww_srce_batch_va: SIZE(VA,1) != NSPEC or NPTS > NSEALM");
      return;
    }
    for (int k = 0; k < npts; ++k) {
      if (jsea[k] < 1 || jsea[k] > nsealm) {
        g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_srce_batch_va: a JSEA outside 1..NSEALM");
        return;
      }
    }
    if (npts == 0) {
      g_status.ok();
      return;
    }
    timers::Region t("srce.batch.call");
    float* d_va = nullptr;
    const int rc = va_device(igrid, va, nspec, nsealm, &d_va);
    if (rc != WW_KOKKOS_OK) {
      g_status.fail(rc, "ww_srce_batch_va: the resident VA refused this call");
      return;
    }
    run_batch(igrid, *g, SrceStep{it, inflags24, flogrd57, flogrd58, dtg}, npts, nullptr, d_va,
              jsea, wn1, cg1, pin, psc, whitecap, taubbl, tauice, shave, "ww_srce_batch_va");
    if (g_status.get() == WW_KOKKOS_OK) va_device_written(igrid);
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

void ww_srce(int igrid, int it, int inflags24, int flogrd57, int flogrd58, float* spec,
             const float* wn1, const float* cg1, float d_inp, float u10abs, float u10dir,
             float as, float ice, float dtg, float dair, float coef, float* ustar, float* ustdir,
             float* tauwx, float* tauwy, float* dtdyn, float* fcut, float* tauox, float* tauoy,
             float* tauwix, float* tauwiy, float* tauwnx, float* tauwny, float* phiaw,
             float* charn, float* tws, float* phioc, float* whitecap, float* phibbl,
             float* taubbl, float* tauice, float* phice, float* tauocx, float* tauocy,
             float* wnmean, float* fpi, int* shave) {
  float* const sc[srce::NPSC] = {ustar,  ustdir, tauwx,  tauwy,  dtdyn,  fcut,   tauox,  tauoy,
                                 tauwix, tauwiy, tauwnx, tauwny, phiaw,  charn,  tws,    phioc,
                                 phibbl, phice,  tauocx, tauocy, wnmean, fpi};
  try {
    GridCtx* g = find(igrid, "ww_srce");
    if (g == nullptr) return;
    bool null = !spec || !wn1 || !cg1 || !whitecap || !taubbl || !tauice || !shave;
    for (float* v : sc) null = null || v == nullptr;
    if (null) {
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_srce: a null argument");
      return;
    }
    const float pin[srce::NPIN] = {d_inp, u10abs, u10dir, as, ice, dair, coef};
    float psc[srce::NPSC];
    for (int j = 0; j < srce::NPSC; ++j) psc[j] = *sc[j];
    run_batch(igrid, *g, SrceStep{it, inflags24, flogrd57, flogrd58, dtg}, 1, spec, nullptr,
              nullptr, wn1, cg1, pin, psc, whitecap, taubbl, tauice, shave, "ww_srce");
    if (g_status.get() == WW_KOKKOS_OK)
      for (int j = 0; j < srce::NPSC; ++j) *sc[j] = psc[j];
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

void ww_srce_batch_device(int igrid, int it, int inflags24, int flogrd57, int flogrd58,
                          float dtg, int npts, float* spec, const float* wn1, const float* cg1,
                          const float* pin, float* psc, float* whitecap, float* taubbl,
                          float* tauice, int* shave, void* stream) {
  try {
    GridCtx* g = find(igrid, "ww_srce_batch_device");
    if (g == nullptr) return;
    if (npts < 0 || (npts > 0 && (!spec || !wn1 || !cg1 || !pin || !psc || !whitecap ||
                                  !taubbl || !tauice || !shave))) {
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_srce_batch_device: npts < 0 or a null array");
      return;
    }
    if (npts == 0) {
      g_status.ok();
      return;
    }
    SrceDev host{};
    if (!prepare(igrid, *g, host, "ww_srce_batch_device")) return;
    launch_srce(g->dev, host.L, SrceStep{it, inflags24, flogrd57, flogrd58, dtg}, npts, spec,
                nullptr, wn1, cg1, pin, psc, whitecap, taubbl, tauice, shave, g->work,
                static_cast<cudaStream_t>(stream));
    g_status.ok();
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_srce_autotune(int igrid, int it, int inflags24, int flogrd57, int flogrd58, float dtg,
                     int npts, const float* spec, const float* wn1, const float* cg1,
                     const float* pin, const float* psc, const float* whitecap,
                     const float* taubbl, const float* tauice) {
  try {
    GridCtx* g = find(igrid, "ww_srce_autotune");
    if (g == nullptr) return -1;
    if (npts < 1 || !spec || !wn1 || !cg1 || !pin || !psc || !whitecap || !taubbl || !tauice) {
      g_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_srce_autotune: npts < 1 or a null array");
      return -1;
    }
    SrceDev host{};
    if (!prepare(igrid, *g, host, "ww_srce_autotune")) return -1;
    const pt::SrceLayout& L = host.L;
    const int maxc = srce_max_ctas_per_sm(L);
    // A sample of the caller's points, four times the most CTAs that can be resident, so every
    // candidate runs several points per CTA (the queue's tail is a small part of the time).
    const int sms = runtime().sm_count;
    const int n = std::min(npts, 4 * maxc * sms);
    const size_t ns = static_cast<size_t>(n) * L.nspec, nk = static_cast<size_t>(n) * L.nk;
    struct Buf {
      float* p = nullptr;
      ~Buf() { if (p) cudaFree(p); }
      float* alloc(size_t k) { WWB_CHECK(cudaMalloc(&p, k * sizeof(float))); return p; }
    };
    Buf s0, s1, w, c, pn, q0, q1, wc0, wc1, tb0, tb1, ti0, ti1, sh;
    s0.alloc(ns), s1.alloc(ns), w.alloc(nk), c.alloc(nk), pn.alloc(n * static_cast<size_t>(srce::NPIN));
    q0.alloc(n * static_cast<size_t>(srce::NPSC)), q1.alloc(n * static_cast<size_t>(srce::NPSC));
    wc0.alloc(4 * static_cast<size_t>(n)), wc1.alloc(4 * static_cast<size_t>(n));
    tb0.alloc(2 * static_cast<size_t>(n)), tb1.alloc(2 * static_cast<size_t>(n));
    ti0.alloc(2 * static_cast<size_t>(n)), ti1.alloc(2 * static_cast<size_t>(n));
    sh.alloc(n);
    auto up = [](float* d, const float* h, size_t k) {
      WWB_CHECK(cudaMemcpy(d, h, k * sizeof(float), cudaMemcpyHostToDevice));
    };
    up(s0.p, spec, ns), up(w.p, wn1, nk), up(c.p, cg1, nk), up(pn.p, pin, n * static_cast<size_t>(srce::NPIN));
    up(q0.p, psc, n * static_cast<size_t>(srce::NPSC)), up(wc0.p, whitecap, 4 * static_cast<size_t>(n));
    up(tb0.p, taubbl, 2 * static_cast<size_t>(n)), up(ti0.p, tauice, 2 * static_cast<size_t>(n));
    std::vector<int> cands;
    for (int k = maxc; k >= 1; --k) cands.push_back(k);
    cudaStream_t st = runtime().stream;
    const SrceStep step{it, inflags24, flogrd57, flogrd58, dtg};
    auto d2d = [&](float* d, const float* s_, size_t k, cudaStream_t ss) {
      WWB_CHECK(cudaMemcpyAsync(d, s_, k * sizeof(float), cudaMemcpyDeviceToDevice, ss));
    };
    const std::string key = "srce ctas/SM " + std::to_string(L.nk) + "x" + std::to_string(L.nth) +
                            " " + tune::device_key();
    const int best = tune::pick(
        key, cands,
        [&](int ctas, cudaStream_t ss) {
          launch_srce(g->dev, L, step, n, s1.p, nullptr, w.p, c.p, pn.p, q1.p, wc1.p, tb1.p, ti1.p,
                      reinterpret_cast<int*>(sh.p), g->work, ss);
          (void)ctas;
        },
        [&](int ctas, cudaStream_t ss) {
          // the candidate's CTAs and carveout, and the sample's inputs restored (W3SRCE updates
          // them in place)
          WWB_CHECK(cudaStreamSynchronize(ss));
          srce_set_ctas_per_sm(L, ctas);
          srce_reserve(L, n, g->work, ss);
          d2d(s1.p, s0.p, ns, ss), d2d(q1.p, q0.p, n * static_cast<size_t>(srce::NPSC), ss);
          d2d(wc1.p, wc0.p, 4 * static_cast<size_t>(n), ss);
          d2d(tb1.p, tb0.p, 2 * static_cast<size_t>(n), ss);
          d2d(ti1.p, ti0.p, 2 * static_cast<size_t>(n), ss);
        },
        st, 2);
    WWB_CHECK(cudaStreamSynchronize(st));
    srce_set_ctas_per_sm(L, best == maxc ? 0 : best);
    g_status.ok();
    return best;
  } catch (const std::exception& e) {
    g_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
    return -1;
  }
}

int ww_srce_enabled(void) { return ww_kokkos_flag("WW_KOKKOS_SRCE") != 0 ? 1 : 0; }

int ww_srce_last_error(void) { return g_status.get(); }

}  // extern "C"
