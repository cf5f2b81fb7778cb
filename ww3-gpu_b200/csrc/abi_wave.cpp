// ww3-gpu_b200/csrc/abi_wave.cpp
// The C ABI of W3WAVE's per-step support routines: ww_wave_gath, ww_wave_scat, ww_wave_uwnd,
// ww_wave_utrn, ww_wave_dzxy, ww_wave_map3, ww_wave_mapt and ww_wave_distab, with the
// reference's names, argument lists and status codes (ww3-gpu
// kokkos/src/fortran_iface/ww_kokkos_c.hpp:893-921; argument tables and checks in
// wave_support_shim.cpp:233-624). No per-grid state: every call carries its sizes, copies its
// arrays in and its results out, as the reference's device path does. W3UTRN, W3MAP3 and W3MAPT
// run the kernels of ww_utrn, ww_map3 and ww_mapt (MAPSF(MSEA,3) compacted to its first NSEA
// rows); the others run wave_kernel.cu. WW_KOKKOS_WAVE_COUNT=1 prints "ww_kokkos: W3<R> calls: N"
// per routine at exit.
//
// ww_wave_cflxy (W3CFLXY) has no entry in the reference's C ABI: there the device W3WAVE driver
// calls it (wave_w3wave.hpp:548-574). Its argument list follows the other routines' (sizes, then
// the module arrays), and like the _va propagation calls it is recorded into grid igrid's step
// while that grid records one.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "staging.hpp"
#include "step.hpp"
#include "wave_kernel.cuh"
#include "wwb_common.hpp"

namespace wwb {
namespace {

enum Routine { GATH, SCAT, UWND, UTRN, DZXY, MAP3, MAPT, DISTAB, CFLXY, NROUTINES };
const char* const kName[NROUTINES] = {"W3GATH", "W3SCAT", "W3UWND", "W3UTRN", "W3DZXY",
                                      "W3MAP3", "W3MAPT", "DISTAB", "W3CFLXY"};
std::atomic<long long> g_calls[NROUTINES];

void print_counts() {
  for (int r = 0; r < NROUTINES; ++r)
    std::fprintf(stderr, "ww_kokkos: %s calls: %lld\n", kName[r], g_calls[r].load());
}

/// One call of routine r; registers the exit print once when WW_KOKKOS_WAVE_COUNT=1.
void count(Routine r) {
  static const bool on = [] {
    const char* v = std::getenv("WW_KOKKOS_WAVE_COUNT");
    const bool c = v != nullptr && std::strcmp(v, "1") == 0;
    if (c) std::atexit(print_counts);
    return c;
  }();
  (void)on;
  g_calls[r].fetch_add(1, std::memory_order_relaxed);
}

int fail(int code, const char* what) {
  std::fprintf(stderr, "ww_b200: W3WAVE support: %s (code %d)\n", what, code);
  return code;
}

Staging& staging() {
  static auto* s = new Staging();
  return *s;
}

/// Runs f() (which returns a status) when the library is initialised; counts a success.
template <class F>
int run(Routine r, F&& f) {
  try {
    if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
    const int rc = f();
    if (rc == WW_KOKKOS_OK) count(r);
    return rc;
  } catch (const std::bad_alloc& e) {
    return fail(WW_KOKKOS_ERR_RUNTIME, e.what());
  } catch (const std::exception& e) {
    return fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

/// MAPSF(MSEA,3)'s first NSEA rows as MAPSF(NSEA,3).
std::vector<int> compact_mapsf(const int* mapsf, int nsea, int msea) {
  std::vector<int> m(3 * static_cast<size_t>(nsea));
  for (int k = 0; k < 3; ++k)
    std::memcpy(m.data() + static_cast<size_t>(k) * nsea, mapsf + static_cast<size_t>(k) * msea,
                sizeof(int) * static_cast<size_t>(nsea));
  return m;
}

/// MAPSF(ISEA,3), ISEA = 1..nsea, all inside the NX*NY cells.
bool ixy_ok(const int* mapsf, int nsea, int msea, long long ncell) {
  const int* ixy = mapsf + 2 * static_cast<size_t>(msea);
  for (int i = 0; i < nsea; ++i)
    if (ixy[i] < 1 || ixy[i] > ncell) return false;
  return true;
}

template <class T>
void d2h(T* h, const T* d, size_t n, cudaStream_t s) {
  if (n) WWB_CHECK(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
}

}  // namespace

void release_wave_staging() { staging().release(); }

}  // namespace wwb

using namespace wwb;

extern "C" {

int ww_wave_gath(int ispec, int nspec, int nsea, int ncol, int msea, int nx, int ny,
                 const float* va, const int* mapsf, float* field) {
  if (ispec < 1 || ispec > nspec || nsea < 0 || ncol < nsea + 1 || msea < nsea || nx < 1 ||
      ny < 1 || va == nullptr || mapsf == nullptr || field == nullptr)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_gath: bad sizes or null pointer");
  if (!ixy_ok(mapsf, nsea, msea, static_cast<long long>(nx) * ny))
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_gath: MAPSF(:,3) outside the grid");
  return run(GATH, [&] {
    const size_t nf = static_cast<size_t>(ny) * (static_cast<size_t>(nx) + 3);
    const size_t n1 = static_cast<size_t>(nsea) + 1, ns = static_cast<size_t>(nspec);
    // The row VA(ISPEC, 0:NSEA): O(NSEA) on the host, as the reference's device path.
    std::vector<float> row(n1);
    for (size_t i = 0; i < n1; ++i) row[i] = va[i * ns + static_cast<size_t>(ispec - 1)];
    Staging& st = staging();
    cudaStream_t s = runtime().stream;
    const float* d_row = st.in(0, row.data(), n1, s);
    const int* d_ixy =
        st.in(1, mapsf + 2 * static_cast<size_t>(msea), static_cast<size_t>(nsea), s);
    float* d_field = static_cast<float*>(st.get(2, nf * sizeof(float)));
    launch_wave_gath(nsea, ny, nf, d_row, d_ixy, d_field, s);
    d2h(field, d_field, nf, s);
    WWB_CHECK(cudaStreamSynchronize(s));
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_wave_scat(int ispec, int nspec, int nsea, int ncol, int msea, int nx, int ny,
                 const int* mapsta, const float* field, const int* mapsf, float* va) {
  if (ispec < 1 || ispec > nspec || nsea < 0 || ncol < nsea + 1 || msea < nsea || nx < 1 ||
      ny < 1 || va == nullptr || mapsf == nullptr || field == nullptr || mapsta == nullptr)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_scat: bad sizes or null pointer");
  if (!ixy_ok(mapsf, nsea, msea, static_cast<long long>(nx) * ny))
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_scat: MAPSF(:,3) outside the grid");
  return run(SCAT, [&] {
    const size_t nf = static_cast<size_t>(ny) * (static_cast<size_t>(nx) + 3);
    const size_t nc = static_cast<size_t>(nx) * ny;
    const size_t n1 = static_cast<size_t>(nsea) + 1, ns = static_cast<size_t>(nspec);
    std::vector<float> row(n1);
    for (size_t i = 0; i < n1; ++i) row[i] = va[i * ns + static_cast<size_t>(ispec - 1)];
    Staging& st = staging();
    cudaStream_t s = runtime().stream;
    float* d_row = st.in(3, row.data(), n1, s);
    const int* d_ixy =
        st.in(4, mapsf + 2 * static_cast<size_t>(msea), static_cast<size_t>(nsea), s);
    const int* d_sta = st.in(5, mapsta, nc, s);
    const float* d_field = st.in(6, field, nf, s);
    launch_wave_scat(nsea, ny, d_sta, d_field, d_ixy, d_row, s);
    d2h(row.data(), d_row, n1, s);
    WWB_CHECK(cudaStreamSynchronize(s));
    for (size_t i = 1; i < n1; ++i) va[i * ns + static_cast<size_t>(ispec - 1)] = row[i];
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_wave_uwnd(int flfrst, float dt0n, float dt0t, int flcur, float rwindc, int nsea, int msea,
                 int nx, int ny, const int* mapsf, const float* wx0, const float* wy0,
                 const float* dt0, const float* wxn, const float* wyn, const float* dtn,
                 const float* cx, const float* cy, float* ua0, float* uai, float* ud0,
                 float* udi, float* as0, float* asi, float* ua, float* ud, float* as,
                 float* u10, float* u10d) {
  if (nsea < 1 || msea < nsea || nx < 1 || ny < 1 || !mapsf || !wx0 || !wy0 || !dt0 || !wxn ||
      !wyn || !dtn || !cx || !cy || !ua0 || !uai || !ud0 || !udi || !as0 || !asi || !ua || !ud ||
      !as || !u10 || !u10d)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_uwnd: bad sizes or null pointer");
  if (flfrst)
    for (int i = 0; i < nsea; ++i)
      if (mapsf[i] < 1 || mapsf[i] > nx || mapsf[msea + i] < 1 || mapsf[msea + i] > ny)
        return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_uwnd: MAPSF names a cell outside the grid");
  return run(UWND, [&] {
    Staging& st = staging();
    cudaStream_t s = runtime().stream;
    const size_t n = static_cast<size_t>(nsea), nc = static_cast<size_t>(nx) * ny;
    UwndArgs a{};
    a.nsea = nsea;
    a.msea = msea;
    a.nx = nx;
    a.ny = ny;
    a.flfrst = flfrst != 0;
    a.flcur = flcur != 0;
    // :684 (WNT1) on the host: RD = DT0T / MAX(1.E-7, DT0N), MAX as the build's maxss.
    a.rd = dt0t / ((dt0n > 1.E-7f) ? dt0n : 1.E-7f);
    a.rwindc = rwindc;
    int k = 10;
    a.mapsf = st.in(k++, mapsf, 3 * static_cast<size_t>(msea), s);
    a.wx0 = st.in(k++, wx0, nc, s);
    a.wy0 = st.in(k++, wy0, nc, s);
    a.dt0 = st.in(k++, dt0, nc, s);
    a.wxn = st.in(k++, wxn, nc, s);
    a.wyn = st.in(k++, wyn, nc, s);
    a.dtn = st.in(k++, dtn, nc, s);
    a.cx = st.in(k++, cx, n, s);
    a.cy = st.in(k++, cy, n, s);
    float* const io[11] = {ua0, uai, ud0, udi, as0, asi, ua, ud, as, u10, u10d};
    float* d[11];
    // UA0..ASI are read without FLFRST: every array comes in.
    for (int j = 0; j < 11; ++j) d[j] = st.in(k++, io[j], n, s);
    a.ua0 = d[0];
    a.uai = d[1];
    a.ud0 = d[2];
    a.udi = d[3];
    a.as0 = d[4];
    a.asi = d[5];
    a.ua = d[6];
    a.ud = d[7];
    a.as = d[8];
    a.u10 = d[9];
    a.u10d = d[10];
    launch_wave_uwnd(a, s);
    for (int j = 0; j < 11; ++j) d2h(io[j], d[j], n, s);
    WWB_CHECK(cudaStreamSynchronize(s));
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_wave_utrn(int nx, int ny, int nsea, int msea, int trflag, float fice0, float ficen,
                 float ficel, float ffacberg, int flagll, const float* trnx, const float* trny,
                 const int* mapsf, const int* mapsta, const float* hpfac, const float* hqfac,
                 const float* ice, const float* berg, float* atrnx, float* atrny) {
  if (nx < 1 || ny < 1 || nsea < 0 || msea < nsea || !trnx || !trny || !mapsf || !mapsta ||
      !hpfac || !hqfac || !ice || !berg || !atrnx || !atrny)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_utrn: bad sizes or null pointer");
  // TRNY(0), the REAL before the array, is read with TRFLAG 1, 3, 5 when cell IXY = 1 is a sea
  // point (w3updtmd.F90:2954): the same address the Fortran reads, only in that case.
  float trny_before = 0.0f;
  if (trflag == 1 || trflag == 3 || trflag == 5)
    for (int i = 0; i < nsea; ++i)
      if (mapsf[2 * static_cast<size_t>(msea) + i] == 1) {
        trny_before = trny[-1];
        break;
      }
  return run(UTRN, [&] {
    const std::vector<int> m = compact_mapsf(mapsf, nsea, msea);
    return ww_utrn(nx, ny, nsea, trflag, fice0, ficen, ficel, ffacberg, flagll, trny_before,
                   trnx, trny, m.data(), mapsta, hpfac, hqfac, ice, berg, atrnx, atrny);
  });
}

int ww_wave_dzxy(int nsea, int nx, int ny, const float* zz, const int* mapsta, const int* mapfs,
                 const float* dpdx, const float* dpdy, const float* dqdx, const float* dqdy,
                 int flagll, int iclose, float* dzzdx, float* dzzdy) {
  if (nsea < 1 || nx < 1 || ny < 1 || !zz || !mapsta || !mapfs || !dpdx || !dpdy || !dqdx ||
      !dqdy || !dzzdx || !dzzdy)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_dzxy: bad sizes or null pointer");
  const size_t nc = static_cast<size_t>(nx) * ny;
  for (size_t c = 0; c < nc; ++c)  // the kernel reads ZZ(MAPFS) at every cell MAPSTA marks sea
    if (mapsta[c] != 0 && (mapfs[c] < 1 || mapfs[c] > nsea))
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_dzxy: MAPFS of a sea cell outside 1..NSEA");
  return run(DZXY, [&] {
    Staging& st = staging();
    cudaStream_t s = runtime().stream;
    DzxyArgs a{};
    a.nx = nx;
    a.ny = ny;
    a.iclose = iclose;
    a.dfac = flagll ? 0x1.2dfd6ap-17f : 1.0f;  // 1./(DERA*RADIUS) as gfortran folds it
    int k = 30;
    a.zz = st.in(k++, zz, static_cast<size_t>(nsea), s);
    a.mapsta = st.in(k++, mapsta, nc, s);
    a.mapfs = st.in(k++, mapfs, nc, s);
    a.dpdx = st.in(k++, dpdx, nc, s);
    a.dpdy = st.in(k++, dpdy, nc, s);
    a.dqdx = st.in(k++, dqdx, nc, s);
    a.dqdy = st.in(k++, dqdy, nc, s);
    a.dzzdx = static_cast<float*>(st.get(k++, nc * sizeof(float)));
    a.dzzdy = static_cast<float*>(st.get(k++, nc * sizeof(float)));
    launch_wave_dzxy(a, s);
    d2h(dzzdx, a.dzzdx, nc, s);
    d2h(dzzdy, a.dzzdy, nc, s);
    WWB_CHECK(cudaStreamSynchronize(s));
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_wave_cflxy(int igrid, int nsea, int msea, int nx, int ny, int nk, int nth, int flcur,
                  int mgp, float dtg, float vgx, float vgy, const int* mapsf, const float* clats,
                  const float* ecos, const float* esin, const float* dpdx, const float* dpdy,
                  const float* dqdx, const float* dqdy, const float* cg, const float* cx,
                  const float* cy, float* cflxymax) {
  if (nsea < 1 || msea < nsea || nx < 1 || ny < 1 || nk < 1 || nth < 1 || nth > 4096 ||
      !mapsf || !clats || !ecos || !esin || !dpdx || !dpdy || !dqdx || !dqdy || !cg ||
      (flcur && (!cx || !cy)) || !cflxymax)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_cflxy: bad sizes or null pointer");
  for (int i = 0; i < nsea; ++i) {  // the kernel reads DPDX..DQDY at (MAPSF(ISEA,1:2))
    const int ix = mapsf[i], iy = mapsf[static_cast<size_t>(msea) + i];
    if (ix < 1 || ix > nx || iy < 1 || iy > ny)
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_cflxy: MAPSF of a sea point off the grid");
  }
  return run(CFLXY, [&] {
    // While grid igrid records a step, the inputs go to buffers the step owns (see step.hpp).
    StepRecorder* const rec = igrid > 0 ? step_recorder(igrid) : nullptr;
    std::shared_ptr<Staging> own = rec ? std::make_shared<Staging>() : nullptr;
    Staging& st = rec ? *own : staging();
    cudaStream_t s = rec ? step_stream(rec) : runtime().stream;
    const size_t nc = static_cast<size_t>(nx) * ny, n1 = static_cast<size_t>(nsea) + 1;
    CflxyArgs a{};
    a.nsea = nsea;
    a.msea = msea;
    a.ny = ny;
    a.nk = nk;
    a.nth = nth;
    a.flcur = flcur != 0;
    a.mgp = mgp != 0;
    a.dtg = dtg;
    a.vgx = vgx;
    a.vgy = vgy;
    int k = 60;
    a.mapsf = st.in(k++, mapsf, 2 * static_cast<size_t>(msea), s);
    a.clats = st.in(k++, clats, n1, s);
    a.ecos = st.in(k++, ecos, static_cast<size_t>(nth), s);
    a.esin = st.in(k++, esin, static_cast<size_t>(nth), s);
    a.dpdx = st.in(k++, dpdx, nc, s);
    a.dpdy = st.in(k++, dpdy, nc, s);
    a.dqdx = st.in(k++, dqdx, nc, s);
    a.dqdy = st.in(k++, dqdy, nc, s);
    a.cg = st.in(k++, cg, static_cast<size_t>(nk + 2) * n1, s);
    a.cx = a.flcur ? st.in(k++, cx, n1, s) : nullptr;
    a.cy = a.flcur ? st.in(k++, cy, n1, s) : nullptr;
    a.cflxymax = static_cast<float*>(st.get(72, static_cast<size_t>(nsea) * sizeof(float)));
    if (rec) {
      // CFLXYMAX of the replays stays on the device, as W3KTP3's CFLTHMAX does.
      WWB_CHECK(cudaStreamSynchronize(s));
      step_keep(rec, own);
      step_add(rec, [a](cudaStream_t ss) { launch_wave_cflxy(a, ss); });
      return static_cast<int>(WW_KOKKOS_OK);
    }
    launch_wave_cflxy(a, s);
    d2h(cflxymax, a.cflxymax, static_cast<size_t>(nsea), s);
    WWB_CHECK(cudaStreamSynchronize(s));
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_wave_map3(int nx, int ny, int nsea, int msea, int nk, int nth, int gtype, const int* mapsta,
                 const int* mapsf, int* mapx2, int* mapy2, int* mapaxy, int* mapcxy, int* mapth2,
                 int* mapwn2, int* counts) {
  if (nx < 1 || ny < 1 || nsea < 1 || msea < nsea || nk < 1 || nth < 1 || gtype < 1 ||
      gtype >= 3 || !mapsta || !mapsf || !mapx2 || !mapy2 || !mapaxy || !mapcxy || !mapth2 ||
      !mapwn2 || !counts)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_map3: bad sizes, GTYPE >= 3 or null pointer");
  return run(MAP3, [&] {
    const std::vector<int> m = compact_mapsf(mapsf, nsea, msea);
    return ww_map3(nx, ny, nsea, nk, nth, gtype, mapsta, m.data(), mapx2, mapy2, mapaxy, mapcxy,
                   mapth2, mapwn2, counts);
  });
}

int ww_wave_mapt(int nsea, int msea, int ncell, const int* mapsf, const float* atrnx,
                 const float* atrny, int* maptrn) {
  if (nsea < 0 || msea < nsea || ncell < 1 || !mapsf || !atrnx || !atrny || !maptrn)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_mapt: bad sizes or null pointer");
  return run(MAPT, [&] {
    const std::vector<int> m = compact_mapsf(mapsf, nsea, msea);
    return ww_mapt(ncell, 1, nsea, m.data(), atrnx, atrny, maptrn);
  });
}

int ww_wave_distab(int nar1d, float* ewn1, float* ecg1, int* n1max, float* dsie) {
  constexpr int kNar1d = 121;  // NAR1D, w3dispmd.F90:75
  if (nar1d != kNar1d || !ewn1 || !ecg1 || !n1max || !dsie)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_wave_distab: NAR1D differs from the port's 121");
  return run(DISTAB, [&] {
    // :652-660 on the host in REAL: N1MAX = NAR1D - 1, SIMAX = SQRT(GRAV*DFAC), DSIE =
    // SIMAX / N1MAX, ECG1(0) = SQRT(GRAV); IEEE sqrt and divide give the folded bits.
    const float grav = 9.806f, dfac = 6.0f;
    const int n1 = kNar1d - 1;
    const float simax = std::sqrt(grav * dfac);
    const float ds = simax / static_cast<float>(n1);
    const float ecg0 = std::sqrt(grav);
    const size_t n = static_cast<size_t>(nar1d) + 1;
    Staging& st = staging();
    cudaStream_t s = runtime().stream;
    float* d_w = static_cast<float*>(st.get(50, n * sizeof(float)));
    float* d_c = static_cast<float*>(st.get(51, n * sizeof(float)));
    launch_wave_distab(nar1d, ds, ecg0, d_w, d_c, s);
    // The caller's arrays hold the Fortran DISTAB's tables: count the values that change.
    std::vector<float> fw(ewn1, ewn1 + n), fc(ecg1, ecg1 + n);
    d2h(ewn1, d_w, n, s);
    d2h(ecg1, d_c, n, s);
    WWB_CHECK(cudaStreamSynchronize(s));
    long long diff = 0;
    for (size_t i = 0; i < n; ++i) {
      if (std::memcmp(&fw[i], &ewn1[i], sizeof(float)) != 0) ++diff;
      if (std::memcmp(&fc[i], &ecg1[i], sizeof(float)) != 0) ++diff;
    }
    if (std::memcmp(&ds, dsie, sizeof(float)) != 0) ++diff;
    if (n1 != *n1max) ++diff;
    std::fprintf(stderr,
                 "ww_kokkos: DISTAB tables rebuilt on the device: %lld of EWN1, ECG1(0:%d), DSIE, "
                 "N1MAX differ from the Fortran's\n",
                 diff, nar1d);
    *n1max = n1;
    *dsie = ds;
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

}  // extern "C"
