// ww3-gpu_b200/csrc/abi_prop3.cpp
// The PR3/UQ half of the C ABI: ww_ktp3_batch and ww_ktp3_batch_va (W3KTP3 for every point of
// one intra-spectral part), and ww_xyp3_batch / ww_xyp3_batch_va (W3XYP3 for every spectral
// component of a propagation step).
//
// Reference: ww3-gpu kokkos/src/fortran_iface/prop3_c.hpp:16-94 and prop3_shim.cpp:835-1068
// (packet lengths, the validation and its order, status codes, the _va forms working on the
// resident VA, whose state is DEVICE afterwards).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <new>

#include "ktp3_kernel.cuh"
#include "staging.hpp"
#include "va.hpp"
#include "wwb_common.hpp"

namespace wwb {
namespace {

Status g_prop3;
Staging& staging() {
  static auto* s = new Staging();
  return *s;
}

int fail(int code, const char* what) { return g_prop3.fail(code, what); }

constexpr int kKtp3NRpar = 3, kKtp3NIpar = 7, kKtp3NPscal = 10;

int ktp3_entry(int igrid, bool resident, const float* rpar, int nrpar, const int* ipar,
               int nipar, const float* sig, const float* dsip, const float* ecos,
               const float* esin, const float* ec2, const float* esc, const float* es2,
               const int* mapwn, const int* mapth2, const int* mapwn2, int itstep, int ntimes,
               float facth, float fack, int nsea, const float* cg, const float* wn, int npts,
               const int* jsea, const int* isea, const float* pscal, int ncol, float* va,
               int nspec_va, int nsealm, float* cflthmax, float* cflkmax) {
  if (rpar == nullptr || ipar == nullptr || nrpar != kKtp3NRpar || nipar != kKtp3NIpar)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_ktp3_batch: bad packet");
  Ktp3Dev p{};
  p.dmin = rpar[0];
  p.ctmax = rpar[1];
  p.fachfa = rpar[2];
  p.nk = ipar[0];
  p.nth = ipar[1];
  p.nspec = ipar[2];
  p.nk2 = ipar[3];
  p.flcth = ipar[4];
  p.flck = ipar[5];
  p.flcur = ipar[6];
  if (p.nk < 1 || p.nth < 1 || p.nspec != p.nk * p.nth || p.nk2 != p.nk + 2 || nsea < 1 ||
      npts < 0 || npts > nsea || ntimes < 0 || ncol < 2 || !sig || !dsip || !ecos || !esin ||
      !ec2 || !esc || !es2 || !mapwn || !mapth2 || !mapwn2 || !cg || !wn || !va || !cflthmax ||
      !cflkmax || (npts > 0 && (!jsea || !isea || !pscal)) || (resident && nspec_va != p.nspec))
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_ktp3_batch: bad sizes or null pointer");
  for (int j = 0; j < npts; ++j)
    if (jsea[j] < 1 || jsea[j] >= ncol || isea[j] < 1 || isea[j] > nsea)
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_ktp3_batch: a point outside VA or the sea");
  // The maps index the work arrays: every entry must stay inside them.
  const int nk2 = p.nk2, nth = p.nth, nspec = p.nspec;
  for (int i = 0; i < nspec; ++i)
    if (mapth2[i] < 1 || mapth2[i] > nk2 * nth || mapwn[i] < 1 || mapwn[i] > p.nk)
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_ktp3_batch: MAPTH2 or MAPWN out of range");
  for (int i = 0; i < nspec + nth; ++i)
    if (mapwn2[i] < 1 || mapwn2[i] > nk2 * nth)
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_ktp3_batch: MAPWN2 out of range");
  if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
  if (ntimes == 0 || npts == 0) {
    g_prop3.ok();
    return WW_KOKKOS_OK;
  }
  timers::Region t_call("ktp3.call");
  Staging& st = staging();
  cudaStream_t s = runtime().stream;
  const size_t ntab = static_cast<size_t>(nspec) + nth;
  const size_t ncell = static_cast<size_t>(nk2) * (static_cast<size_t>(nsea) + 1);
  const size_t ncfl = static_cast<size_t>(ncol) - 1;
  int slot = 0;
  p.sig = st.in(slot++, sig, nk2, s);
  p.dsip = st.in(slot++, dsip, nk2, s);
  p.ecos = st.in(slot++, ecos, ntab, s);
  p.esin = st.in(slot++, esin, ntab, s);
  p.ec2 = st.in(slot++, ec2, ntab, s);
  p.esc = st.in(slot++, esc, ntab, s);
  p.es2 = st.in(slot++, es2, ntab, s);
  p.mapwn = st.in(slot++, mapwn, ntab, s);
  p.mapth2 = st.in(slot++, mapth2, static_cast<size_t>(nk2) * nth, s);
  p.mapwn2 = st.in(slot++, mapwn2, ntab, s);
  const float* d_cg = st.in(slot++, cg, ncell, s);
  const float* d_wn = st.in(slot++, wn, ncell, s);
  const int* d_js = st.in(slot++, jsea, static_cast<size_t>(npts), s);
  const int* d_is = st.in(slot++, isea, static_cast<size_t>(npts), s);
  const float* d_ps = st.in(slot++, pscal, static_cast<size_t>(kKtp3NPscal) * npts, s);
  float* d_va = nullptr;
  if (resident) {
    const int rc = va_device(igrid, va, nspec_va, nsealm, &d_va);
    if (rc != WW_KOKKOS_OK) return fail(rc, "ww_ktp3_batch_va: the resident VA refused this call");
  } else {
    d_va = st.in(slot++, va, static_cast<size_t>(nspec) * ncol, s);
  }
  // CFLTHMAX/CFLKMAX come in as well as out: entries of points not listed keep their values.
  float* d_cth = st.in(slot++, cflthmax, ncfl, s);
  float* d_ck = st.in(slot++, cflkmax, ncfl, s);
  launch_ktp3(p, itstep, ntimes, facth, fack, npts, d_js, d_is, d_ps, d_cg, d_wn, d_va, d_cth,
              d_ck, s);
  if (resident) va_device_written(igrid);
  else
    WWB_CHECK(cudaMemcpyAsync(va, d_va, sizeof(float) * nspec * static_cast<size_t>(ncol),
                              cudaMemcpyDeviceToHost, s));
  WWB_CHECK(cudaMemcpyAsync(cflthmax, d_cth, sizeof(float) * ncfl, cudaMemcpyDeviceToHost, s));
  WWB_CHECK(cudaMemcpyAsync(cflkmax, d_ck, sizeof(float) * ncfl, cudaMemcpyDeviceToHost, s));
  WWB_CHECK(cudaStreamSynchronize(s));
  g_prop3.ok();
  return WW_KOKKOS_OK;
}

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc& e) {
    return fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  } catch (const std::exception& e) {
    return fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

}  // namespace

void release_prop3_staging() { staging().release(); }

}  // namespace wwb

using namespace wwb;

extern "C" {

int ww_ktp3_batch(const float* rpar, int nrpar, const int* ipar, int nipar, const float* sig,
                  const float* dsip, const float* ecos, const float* esin, const float* ec2,
                  const float* esc, const float* es2, const int* mapwn, const int* mapth2,
                  const int* mapwn2, int itstep, int ntimes, float facth, float fack, int nsea,
                  const float* cg, const float* wn, int npts, const int* jsea, const int* isea,
                  const float* pscal, int ncol, float* va, float* cflthmax, float* cflkmax) {
  return guarded([&] {
    return ktp3_entry(0, false, rpar, nrpar, ipar, nipar, sig, dsip, ecos, esin, ec2, esc, es2,
                      mapwn, mapth2, mapwn2, itstep, ntimes, facth, fack, nsea, cg, wn, npts,
                      jsea, isea, pscal, ncol, va, 0, 0, cflthmax, cflkmax);
  });
}

int ww_ktp3_batch_va(int igrid, const float* rpar, int nrpar, const int* ipar, int nipar,
                     const float* sig, const float* dsip, const float* ecos, const float* esin,
                     const float* ec2, const float* esc, const float* es2, const int* mapwn,
                     const int* mapth2, const int* mapwn2, int itstep, int ntimes, float facth,
                     float fack, int nsea, const float* cg, const float* wn, int npts,
                     const int* jsea, const int* isea, const float* pscal, float* va, int nspec,
                     int nsealm, float* cflthmax, float* cflkmax) {
  return guarded([&] {
    return ktp3_entry(igrid, true, rpar, nrpar, ipar, nipar, sig, dsip, ecos, esin, ec2, esc,
                      es2, mapwn, mapth2, mapwn2, itstep, ntimes, facth, fack, nsea, cg, wn,
                      npts, jsea, isea, pscal, nsealm + 1, va, nspec, nsealm, cflthmax,
                      cflkmax);
  });
}

int ww_prop3_last_error(void) { return g_prop3.get(); }

}  // extern "C"
