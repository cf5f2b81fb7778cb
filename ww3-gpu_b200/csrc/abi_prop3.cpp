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
#include <algorithm>
#include <cstdlib>
#include <cstdint>
#include <new>
#include <vector>

#include "ktp3_kernel.cuh"
#include "map3_kernel.cuh"
#include "staging.hpp"
#include "step.hpp"
#include "utrn_kernel.cuh"
#include "va.hpp"
#include "wwb_common.hpp"
#include "xyp3_kernel.cuh"

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
  // While the grid records a step, the inputs go to buffers the step owns (see step.hpp).
  StepRecorder* const rec = resident ? step_recorder(igrid) : nullptr;
  std::shared_ptr<Staging> own = rec ? std::make_shared<Staging>() : nullptr;
  Staging& st = rec ? *own : staging();
  cudaStream_t s = rec ? step_stream(rec) : runtime().stream;
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
  if (rec) {
    // CFLTHMAX/CFLKMAX of the replays stay on the device.
    WWB_CHECK(cudaStreamSynchronize(s));
    step_keep(rec, own);
    step_add(rec, [=](cudaStream_t ss) {
      launch_ktp3(p, itstep, ntimes, facth, fack, npts, d_js, d_is, d_ps, d_cg, d_wn, d_va,
                  d_cth, d_ck, ss);
    });
    g_prop3.ok();
    return WW_KOKKOS_OK;
  }
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

constexpr int kXyp3NRpar = 5, kXyp3NIpar = 11, kXyp3NImaps = 8, kXyp3NTscal = 3;
constexpr int kIcloseNone = -1, kIcloseTrpl = 8;
/// Work storage of one XYP3 chunk is capped so a call never asks for more than this.
constexpr size_t kXyp3ChunkBytes = size_t(8) << 30;

struct Xyp3Args {
  const float *rpar, *tscal, *clats, *sig, *ecos, *esin, *dpdx, *dpdy, *dqdx, *dqdy, *gsqrt;
  const float *atrnx, *atrny, *cg, *cx, *cy, *bbpi0, *bbpin;
  const int *ipar, *imaps, *mapsf, *mapx2, *mapy2, *mapaxy, *mapcxy, *maptrn, *mapsta, *isbpi,
      *on;
  int nrpar, nipar, nimaps, ntscal, flbpi, nbi, ncol;
  float dtg;
  float* va;
  // ww_xyp3_batch_mpi only (naproc > 0): the ranks, the offsets of the other ranks' blocks, the
  // received values (GSTORE) and the values to send back (SSTORE), nbuf floats each.
  int naproc = 0, iaproc = 0, nbuf = 0;
  const int* poff = nullptr;
  const float* rbuf = nullptr;
  float* sbuf = nullptr;
};

int xyp3_entry(int igrid, bool resident, const Xyp3Args& a, int nspec_va, int nsealm) {
  if (!a.rpar || !a.ipar || !a.imaps || !a.tscal || a.nrpar != kXyp3NRpar ||
      a.nipar != kXyp3NIpar || a.nimaps != kXyp3NImaps || a.ntscal != kXyp3NTscal)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch: bad packet");
  Xyp3Grid g{};
  g.dtcfl = a.rpar[0];
  g.dth = a.rpar[1];
  g.xfr = a.rpar[2];
  g.wdcg = a.rpar[3];
  g.wdth = a.rpar[4];
  g.nx = a.ipar[0];
  g.ny = a.ipar[1];
  g.nsea = a.ipar[2];
  g.nk = a.ipar[3];
  g.nth = a.ipar[4];
  g.nspec = a.ipar[5];
  g.iclose = a.ipar[6];
  g.flcx = a.ipar[7];
  g.flcy = a.ipar[8];
  g.flagll = a.ipar[9];
  g.flcur = a.ipar[10];
  if (g.nx < 1 || g.ny < 1 || g.nsea < 1 || g.nk < 1 || g.nth < 1 || g.nspec != g.nk * g.nth ||
      (a.naproc == 0 && a.ncol < g.nsea + 1) || a.nbi < 0 || !a.mapsf || !a.clats || !a.sig || !a.ecos || !a.esin ||
      !a.dpdx || !a.dpdy || !a.dqdx || !a.dqdy || !a.gsqrt || !a.atrnx || !a.atrny ||
      !a.mapx2 || !a.mapy2 || !a.mapaxy || !a.mapcxy || !a.maptrn || !a.mapsta || !a.cg ||
      !a.cx || !a.cy || !a.on || !a.va ||
      (a.flbpi != 0 && (!a.isbpi || !a.bbpi0 || !a.bbpin)) ||
      (resident && nspec_va != g.nspec))
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch: bad sizes or null pointer");
  if (g.iclose == kIcloseTrpl)
    return fail(WW_KOKKOS_ERR_UNSUPPORTED, "ww_xyp3_batch: tripole grid (W3XYP3 stops there)");
  int nsploc = 0;
  for (int isp = 0; isp < g.nspec; ++isp) nsploc += a.on[isp] != 0 ? 1 : 0;
  if (a.naproc != 0) {
    // Every sea point is some rank's column K <= NSEALM, and every other rank's block holds this
    // rank's NSPLOC components of NSEALM values each, in rank order (prop3_shim.cpp:793-811).
    const long long nsealm_ll = a.ncol - 1;
    if (!resident || a.naproc < 1 || a.iaproc < 1 || a.iaproc > a.naproc || nsealm_ll < 1 ||
        nsealm_ll * a.naproc < g.nsea || !a.poff ||
        a.nbuf != static_cast<long long>(a.naproc - 1) * nsploc * nsealm_ll ||
        (a.nbuf > 0 && (!a.rbuf || !a.sbuf)))
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch_mpi: bad ranks, offsets or buffers");
    for (int ip = 1, off = 0; ip <= a.naproc; ++ip) {
      if (ip == a.iaproc) continue;
      if (a.poff[ip - 1] != off)
        return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch_mpi: offsets not in rank order");
      off += nsploc * static_cast<int>(nsealm_ll);
    }
  }
  g.global = g.iclose != kIcloseNone ? 1 : 0;
  if (g.global && g.nx < 3)
    return fail(WW_KOKKOS_ERR_UNSUPPORTED, "ww_xyp3_batch: a closed grid needs NX >= 3");
  g.nmx0 = a.imaps[0];
  g.nmx1 = a.imaps[1];
  g.nmx2 = a.imaps[2];
  g.nmy0 = a.imaps[3];
  g.nmy1 = a.imaps[4];
  g.nmy2 = a.imaps[5];
  g.nact = a.imaps[6];
  g.ncent = a.imaps[7];
  const int nx = g.nx, ny = g.ny, nsea = g.nsea, nxy = nx * ny;
  // Every map entry must address the arrays the kernels hold.
  auto bad_counts = [&](int c0, int c1, int c2) { return c0 < 0 || c1 < c0 || c2 < c1 || c2 > nxy; };
  if (bad_counts(g.nmx0, g.nmx1, g.nmx2) || bad_counts(g.nmy0, g.nmy1, g.nmy2) || g.nact < 0 ||
      g.nact > nxy || g.ncent < 0 || g.ncent > nsea)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch: map counts out of range");
  for (int i = 0; i < g.nmx2; ++i)
    if (a.mapx2[i] < 1 || a.mapx2[i] > nxy) return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch: MAPX2 out of range");
  for (int i = 0; i < g.nmy2; ++i)
    if (a.mapy2[i] < 1 || a.mapy2[i] > nxy) return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch: MAPY2 out of range");
  for (int i = 0; i < g.nact; ++i)
    if (a.mapaxy[i] < 1 || a.mapaxy[i] > nxy) return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch: MAPAXY out of range");
  std::vector<int> cell_sea(nxy, 0), sea_pos(nsea, 0), bnd_last(nsea, 0);
  for (int isea = 1; isea <= nsea; ++isea) {
    const int ix = a.mapsf[isea - 1], iy = a.mapsf[nsea + isea - 1], ixy = a.mapsf[2 * nsea + isea - 1];
    if (ix < 1 || ix > nx || iy < 1 || iy > ny || ixy != (ix - 1) * ny + iy || cell_sea[ixy - 1] != 0)
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch: MAPSF is not a map of sea cells");
    cell_sea[ixy - 1] = isea;
  }
  for (int ip = 1; ip <= nsea; ++ip) {
    const int isea = a.mapcxy[ip - 1];
    if (isea < 1 || isea > nsea || sea_pos[isea - 1] != 0)
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch: MAPCXY is not a permutation");
    sea_pos[isea - 1] = ip;
  }
  const int nbi = a.flbpi != 0 ? a.nbi : 0;
  for (int ibi = 1; ibi <= nbi; ++ibi) {
    const int ib = a.isbpi[ibi - 1];
    if (ib < 1 || ib > nsea) return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_batch: ISBPI out of range");
    bnd_last[ib - 1] = ibi;  // the last IBI naming a point wins, as the serial loop's last write
  }
  std::vector<int> mapstx(static_cast<size_t>(ny) * (nx + 4), 0);
  for (int i = 1; i <= nxy; ++i) mapstx[i + 2 * ny - 1] = a.mapsta[i - 1];
  if (g.global)
    for (int j = 0; j < 2 * ny; ++j) {
      mapstx[(1 - 2 * ny + j) + 2 * ny - 1] = a.mapsta[(nx - 2) * ny + j];
      mapstx[(nxy + 1 + j) + 2 * ny - 1] = a.mapsta[j];
    }
  // The dense cell map of the tiled W3QCK3 sweeps (Xyp3Grid::cell_kind).
  std::vector<unsigned char> kind(static_cast<size_t>(nxy), 0);
  bool unique = true;
  auto mark = [&](const int* m, int n0, int n1, int n2, int shift) {
    for (int ip = 1; ip <= n2; ++ip) {
      unsigned char& k = kind[m[ip - 1] - 1];
      if ((k >> shift) & 3) unique = false;
      k = static_cast<unsigned char>(k | ((ip <= n0 ? 1 : ip <= n1 ? 2 : 3) << shift));
    }
  };
  mark(a.mapx2, g.nmx0, g.nmx1, g.nmx2, 0);
  mark(a.mapy2, g.nmy0, g.nmy1, g.nmy2, 2);
  for (int ip = 1; ip <= g.nact; ++ip) {
    unsigned char& k = kind[a.mapaxy[ip - 1] - 1];
    if (k & 16) unique = false;
    k = static_cast<unsigned char>(k | 16);
  }
  std::vector<int> list;
  for (int isp = 1; isp <= g.nspec; ++isp)
    if (a.on[isp - 1] != 0) list.push_back(isp);
  if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
  timers::Region t_call("xyp3.call");
  StepRecorder* const rec = resident ? step_recorder(igrid) : nullptr;
  if (rec && a.naproc != 0)
    return fail(WW_KOKKOS_ERR_UNSUPPORTED, "ww_xyp3_batch_mpi: not recorded into a step");
  std::shared_ptr<Staging> own = rec ? std::make_shared<Staging>() : nullptr;
  Staging& st = rec ? *own : staging();
  cudaStream_t s = rec ? step_stream(rec) : runtime().stream;
  const size_t nk2 = static_cast<size_t>(g.nk) + 2, ntab = static_cast<size_t>(g.nspec) + g.nth;
  int slot = 0;
  g.mapsf = st.in(slot++, a.mapsf, 3 * static_cast<size_t>(nsea), s);
  g.clats = st.in(slot++, a.clats, static_cast<size_t>(nsea) + 1, s);
  g.sig = st.in(slot++, a.sig, nk2, s);
  g.ecos = st.in(slot++, a.ecos, ntab, s);
  g.esin = st.in(slot++, a.esin, ntab, s);
  g.dpdx = st.in(slot++, a.dpdx, static_cast<size_t>(nxy), s);
  g.dpdy = st.in(slot++, a.dpdy, static_cast<size_t>(nxy), s);
  g.dqdx = st.in(slot++, a.dqdx, static_cast<size_t>(nxy), s);
  g.dqdy = st.in(slot++, a.dqdy, static_cast<size_t>(nxy), s);
  g.gsqrt = st.in(slot++, a.gsqrt, static_cast<size_t>(nxy), s);
  g.atrnx = st.in(slot++, a.atrnx, 3 * static_cast<size_t>(nxy), s);
  g.atrny = st.in(slot++, a.atrny, 3 * static_cast<size_t>(nxy), s);
  g.mapx2 = st.in(slot++, a.mapx2, static_cast<size_t>(nxy), s);
  g.mapy2 = st.in(slot++, a.mapy2, static_cast<size_t>(nxy), s);
  g.mapaxy = st.in(slot++, a.mapaxy, static_cast<size_t>(nxy), s);
  g.maptrn = st.in(slot++, a.maptrn, static_cast<size_t>(nxy), s);
  g.mapsta = st.in(slot++, a.mapsta, static_cast<size_t>(nxy), s);
  g.mapstx = st.in(slot++, mapstx.data(), mapstx.size(), s);
  g.cell_sea = st.in(slot++, cell_sea.data(), cell_sea.size(), s);
  g.sea_pos = st.in(slot++, sea_pos.data(), sea_pos.size(), s);
  g.bnd_last = st.in(slot++, bnd_last.data(), bnd_last.size(), s);
  // WW_B200_XYP3_LISTS=1 runs the sweeps as list kernels (the same bits; for comparisons).
  const char* lists = std::getenv("WW_B200_XYP3_LISTS");
  const bool tiled = unique && !(lists != nullptr && std::strcmp(lists, "1") == 0);
  g.cell_kind = tiled ? st.in(slot++, kind.data(), kind.size(), s) : nullptr;
  g.cg = st.in(slot++, a.cg, nk2 * (static_cast<size_t>(nsea) + 1), s);
  g.cx = st.in(slot++, a.cx, static_cast<size_t>(nsea) + 1, s);
  g.cy = st.in(slot++, a.cy, static_cast<size_t>(nsea) + 1, s);
  const size_t nbb = nbi > 0 ? static_cast<size_t>(g.nspec) * (nbi + 1) : 1;
  static const float kZero[1] = {0.0f};
  g.bbpi0 = nbi > 0 ? st.in(slot++, a.bbpi0, nbb, s) : st.in(slot++, kZero, 1, s);
  g.bbpin = nbi > 0 ? st.in(slot++, a.bbpin, nbb, s) : st.in(slot++, kZero, 1, s);
  g.flbpi = a.flbpi != 0 ? 1 : 0;
  g.nbi = nbi;
  g.dsec_day = a.tscal[0];
  g.dsec_bpi0 = a.flbpi != 0 ? a.tscal[1] : 0.0f;
  g.dsec_bpin = a.flbpi != 0 ? a.tscal[2] : 0.0f;
  g.dtg = a.dtg;
  if (g.flcur != 0) xyp3_current_range(g, s);
  if (g.cell_kind != nullptr && ny >= 3) {  // the tiled averaging's source lists (grid only)
    g.gather_order = static_cast<unsigned long long*>(
        st.get(slot++, sizeof(unsigned long long) * static_cast<size_t>(ny) * (nx + 3)));
    launch_xyp3_gather_order(g, s);
  }
  float* d_va = nullptr;
  if (resident) {
    const int rc = va_device(igrid, a.va, nspec_va, nsealm, &d_va);
    if (rc != WW_KOKKOS_OK) return fail(rc, "ww_xyp3_batch_va: the resident VA refused this call");
  } else {
    d_va = st.in(slot++, a.va, static_cast<size_t>(g.nspec) * a.ncol, s);
  }
  const int* d_list = st.in(slot++, list.data(), list.size(), s);
  const size_t nbuf = static_cast<size_t>(a.nbuf);
  if (a.naproc > 0) {
    g.naproc = a.naproc;
    g.iaproc = a.iaproc;
    g.nsealm = a.ncol - 1;
    g.poff = st.in(slot++, a.poff, static_cast<size_t>(a.naproc), s);
    g.rbuf = st.in(slot++, a.rbuf, nbuf, s);
    // SSTORE starts at 0 and W3SCAT writes sea points only: entries past NSEA stay 0.
    g.sbuf = static_cast<float*>(st.get(slot++, nbuf * sizeof(float)));
    if (nbuf > 0) WWB_CHECK(cudaMemsetAsync(g.sbuf, 0, nbuf * sizeof(float), s));
  }
  // Chunks of components, their work arrays carved from one staging slot.
  const size_t per = xyp3_bytes_per_component(g);
  const int chunk = static_cast<int>(std::max<size_t>(1, std::min<size_t>(list.size(), kXyp3ChunkBytes / per)));
  const size_t nq = static_cast<size_t>(ny) * (nx + 3), n1 = static_cast<size_t>(ny) * (nx + 1);
  char* base = static_cast<char*>(st.get(slot++, per * chunk + 256));
  std::vector<std::pair<Xyp3Chunk, int>> recorded;  // chunks and sub-step counts of a step
  for (size_t c0 = 0; c0 < list.size(); c0 += chunk) {
    Xyp3Chunk ch{};
    ch.ncomp = static_cast<int>(std::min<size_t>(chunk, list.size() - c0));
    ch.l0 = static_cast<int>(c0);
    ch.isp = d_list + c0;
    float* f = reinterpret_cast<float*>(base);
    ch.vq = f;
    ch.aq = ch.vq + nq * chunk;
    ch.vlcflx = ch.aq + nq * chunk;
    ch.vlcfly = ch.vlcflx + n1 * chunk;
    ch.fla = ch.vlcfly + n1 * chunk;
    ch.rdi = ch.fla + n1 * chunk;
    ch.iixy = reinterpret_cast<int*>(ch.rdi + 4 * static_cast<size_t>(nsea) * chunk);
    ch.tcode = reinterpret_cast<unsigned*>(ch.iixy + 4 * static_cast<size_t>(nsea) * chunk);
    ch.comp = reinterpret_cast<Comp*>(
        (reinterpret_cast<uintptr_t>(ch.tcode + static_cast<size_t>(nsea) * chunk) + 63) &
        ~static_cast<uintptr_t>(63));
    if (rec) {
      // The chunks share the work arrays (they run one after another); each keeps its own
      // per-component constants.
      ch.comp = static_cast<Comp*>(st.get(slot++, xyp3_comp_bytes() * ch.ncomp));
      const int ntmax = setup_xyp3_chunk(g, ch, s);
      recorded.emplace_back(ch, ntmax);
    } else {
      run_xyp3_chunk(g, ch, d_va, s);
    }
  }
  if (rec) {
    WWB_CHECK(cudaStreamSynchronize(s));
    step_keep(rec, own);
    step_add(rec, [g, recorded, d_va](cudaStream_t ss) {
      for (const auto& cn : recorded) launch_xyp3_chunk(g, cn.first, d_va, cn.second, ss);
    });
    g_prop3.ok();
    return WW_KOKKOS_OK;
  }
  if (resident) va_device_written(igrid);
  else
    WWB_CHECK(cudaMemcpyAsync(a.va, d_va, sizeof(float) * g.nspec * static_cast<size_t>(a.ncol),
                              cudaMemcpyDeviceToHost, s));
  if (a.naproc > 0 && nbuf > 0)
    WWB_CHECK(cudaMemcpyAsync(a.sbuf, g.sbuf, nbuf * sizeof(float), cudaMemcpyDeviceToHost, s));
  WWB_CHECK(cudaStreamSynchronize(s));
  g_prop3.ok();
  return WW_KOKKOS_OK;
}

/// ww_xyp3_mpi_pack (unpack false) and ww_xyp3_mpi_unpack (unpack true) on the resident VA of
/// grid igrid (prop3_shim.cpp:887-925): buf[J*NSEALM + K-1] and VA(ISPS(J+1), K).
int xyp3_mpi_move(bool unpack, int igrid, float* va, int nspec, int nsealm, const int* isps,
                  int nisp, float* buf) {
  if (!va || nspec < 1 || nsealm < 1 || nisp < 0 || nisp > nspec ||
      (nisp > 0 && (!isps || !buf)))
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_mpi_pack/unpack: bad sizes or null pointer");
  for (int j = 0; j < nisp; ++j)
    if (isps[j] < 1 || isps[j] > nspec)
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_xyp3_mpi_pack/unpack: a component outside VA");
  if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
  timers::Region t_call(unpack ? "xyp3.unpack" : "xyp3.pack");
  float* d_va = nullptr;
  const int rc = va_device(igrid, va, nspec, nsealm, &d_va);
  if (rc != WW_KOKKOS_OK)
    return fail(rc, "ww_xyp3_mpi_pack/unpack: the resident VA refused this call");
  const size_t n = static_cast<size_t>(nisp) * nsealm;
  if (n > 0) {
    Staging& st = staging();
    cudaStream_t s = runtime().stream;
    // Slots past the XYP3 call's, so a pack between two steps reuses its own buffers.
    constexpr int kSlot = 64;
    const int* d_isps = st.in(kSlot, isps, static_cast<size_t>(nisp), s);
    float* d_buf = unpack ? st.in(kSlot + 1, static_cast<const float*>(buf), n, s)
                          : static_cast<float*>(st.get(kSlot + 1, n * sizeof(float)));
    launch_va_components(unpack, d_va, nspec, nsealm, d_isps, nisp, d_buf, s);
    if (!unpack)
      WWB_CHECK(cudaMemcpyAsync(buf, d_buf, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    WWB_CHECK(cudaStreamSynchronize(s));
  }
  // A pack only read the device copy; an unpack wrote it.
  if (unpack) va_device_written(igrid);
  g_prop3.ok();
  return WW_KOKKOS_OK;
}

Map3Work& map3_work() {
  static auto* w = new Map3Work();
  return *w;
}

/// W3MAP3's inputs must address the grid: MAPSF's IX, IY in range and IXY = IY + (IX-1)*NY.
int map3_check(int nx, int ny, int nsea, int nk, int nth, const int* mapsta, const int* mapsf,
               const void* mapx2, const void* mapy2, const void* mapaxy, const void* mapcxy,
               const void* mapth2, const void* mapwn2, const void* counts, bool host_mapsf) {
  if (nx < 1 || ny < 1 || nsea < 0 || nk < 1 || nth < 1 ||
      static_cast<long long>(nx) * ny > (1ll << 31) - 1 || !mapsta || (nsea > 0 && !mapsf) ||
      !mapx2 || !mapy2 || !mapaxy || (nsea > 0 && !mapcxy) || !mapth2 || !mapwn2 || !counts)
    return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_map3: bad sizes or null pointer");
  if (host_mapsf)
    for (int i = 0; i < nsea; ++i) {
      const int ix = mapsf[i], iy = mapsf[nsea + i], ixy = mapsf[2 * nsea + i];
      if (ix < 1 || ix > nx || iy < 1 || iy > ny || ixy != (ix - 1) * ny + iy)
        return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_map3: MAPSF is not a map of cells of the grid");
    }
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

void release_prop3_staging() {
  staging().release();
  map3_work().release();
}

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

int ww_xyp3_batch(const float* rpar, int nrpar, const int* ipar, int nipar, const int* imaps,
                  int nimaps, const float* tscal, int ntscal, float dtg, const int* mapsf,
                  const float* clats, const float* sig, const float* ecos, const float* esin,
                  const float* dpdx, const float* dpdy, const float* dqdx, const float* dqdy,
                  const float* gsqrt, const float* atrnx, const float* atrny, const int* mapx2,
                  const int* mapy2, const int* mapaxy, const int* mapcxy, const int* maptrn,
                  const int* mapsta, const float* cg, const float* cx, const float* cy,
                  int flbpi, int nbi, const int* isbpi, const float* bbpi0, const float* bbpin,
                  const int* on, int ncol, float* va) {
  const Xyp3Args a{rpar,  tscal, clats, sig,    ecos,   esin,   dpdx,   dpdy,   dqdx,   dqdy,
                   gsqrt, atrnx, atrny, cg,     cx,     cy,     bbpi0,  bbpin,  ipar,   imaps,
                   mapsf, mapx2, mapy2, mapaxy, mapcxy, maptrn, mapsta, isbpi,  on,     nrpar,
                   nipar, nimaps, ntscal, flbpi, nbi, ncol, dtg, va};
  return guarded([&] { return xyp3_entry(0, false, a, 0, 0); });
}

int ww_xyp3_batch_va(int igrid, const float* rpar, int nrpar, const int* ipar, int nipar,
                     const int* imaps, int nimaps, const float* tscal, int ntscal, float dtg,
                     const int* mapsf, const float* clats, const float* sig, const float* ecos,
                     const float* esin, const float* dpdx, const float* dpdy, const float* dqdx,
                     const float* dqdy, const float* gsqrt, const float* atrnx,
                     const float* atrny, const int* mapx2, const int* mapy2, const int* mapaxy,
                     const int* mapcxy, const int* maptrn, const int* mapsta, const float* cg,
                     const float* cx, const float* cy, int flbpi, int nbi, const int* isbpi,
                     const float* bbpi0, const float* bbpin, const int* on, float* va, int nspec,
                     int nsealm) {
  const Xyp3Args a{rpar,  tscal, clats, sig,    ecos,   esin,   dpdx,   dpdy,   dqdx,   dqdy,
                   gsqrt, atrnx, atrny, cg,     cx,     cy,     bbpi0,  bbpin,  ipar,   imaps,
                   mapsf, mapx2, mapy2, mapaxy, mapcxy, maptrn, mapsta, isbpi,  on,     nrpar,
                   nipar, nimaps, ntscal, flbpi, nbi, nsealm + 1, dtg, va};
  return guarded([&] { return xyp3_entry(igrid, true, a, nspec, nsealm); });
}

int ww_xyp3_batch_mpi(int igrid, const float* rpar, int nrpar, const int* ipar, int nipar,
                      const int* imaps, int nimaps, const float* tscal, int ntscal, float dtg,
                      const int* mapsf, const float* clats, const float* sig, const float* ecos,
                      const float* esin, const float* dpdx, const float* dpdy, const float* dqdx,
                      const float* dqdy, const float* gsqrt, const float* atrnx,
                      const float* atrny, const int* mapx2, const int* mapy2, const int* mapaxy,
                      const int* mapcxy, const int* maptrn, const int* mapsta, const float* cg,
                      const float* cx, const float* cy, int flbpi, int nbi, const int* isbpi,
                      const float* bbpi0, const float* bbpin, const int* on, float* va,
                      int nspec, int nsealm, int naproc, int iaproc, const int* poff,
                      const float* rbuf, float* sbuf, int nbuf) {
  Xyp3Args a{rpar,  tscal, clats, sig,    ecos,   esin,   dpdx,   dpdy,   dqdx,   dqdy,
             gsqrt, atrnx, atrny, cg,     cx,     cy,     bbpi0,  bbpin,  ipar,   imaps,
             mapsf, mapx2, mapy2, mapaxy, mapcxy, maptrn, mapsta, isbpi,  on,     nrpar,
             nipar, nimaps, ntscal, flbpi, nbi, nsealm + 1, dtg, va};
  // naproc < 1 is refused as a bad rank count, not taken for W3_SHRD.
  a.naproc = naproc < 1 ? -1 : naproc;
  a.iaproc = iaproc;
  a.poff = poff;
  a.rbuf = rbuf;
  a.sbuf = sbuf;
  a.nbuf = nbuf;
  return guarded([&] { return xyp3_entry(igrid, true, a, nspec, nsealm); });
}

int ww_xyp3_mpi_pack(int igrid, float* va, int nspec, int nsealm, const int* isps, int nisp,
                     float* buf) {
  return guarded([&] { return xyp3_mpi_move(false, igrid, va, nspec, nsealm, isps, nisp, buf); });
}

int ww_xyp3_mpi_unpack(int igrid, float* va, int nspec, int nsealm, const int* isps, int nisp,
                       const float* buf) {
  return guarded([&] {
    return xyp3_mpi_move(true, igrid, va, nspec, nsealm, isps, nisp, const_cast<float*>(buf));
  });
}

int ww_map3(int nx, int ny, int nsea, int nk, int nth, int gtype, const int* mapsta,
            const int* mapsf, int* mapx2, int* mapy2, int* mapaxy, int* mapcxy, int* mapth2,
            int* mapwn2, int* counts) {
  return guarded([&] {
    if (const int rc = map3_check(nx, ny, nsea, nk, nth, mapsta, mapsf, mapx2, mapy2, mapaxy,
                                  mapcxy, mapth2, mapwn2, counts, true);
        rc != WW_KOKKOS_OK)
      return rc;
    if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
    timers::Region t_call("map3.call");
    Staging& st = staging();
    cudaStream_t s = runtime().stream;
    const size_t nxy = static_cast<size_t>(nx) * ny, nth2 = static_cast<size_t>(nk + 2) * nth,
                 nwn2 = static_cast<size_t>(nk) * nth + nth;
    // Slots past the PR3 calls' own. The maps come in as well as out: entries past the
    // counters keep the caller's values.
    constexpr int k0 = 80;
    const int* d_sta = st.in(k0, mapsta, nxy, s);
    const int* d_sf = st.in(k0 + 1, mapsf, 3 * static_cast<size_t>(nsea), s);
    int* d_x2 = st.in(k0 + 2, mapx2, nxy, s);
    int* d_y2 = st.in(k0 + 3, mapy2, nxy, s);
    int* d_axy = st.in(k0 + 4, mapaxy, nxy, s);
    int* d_cxy = st.in(k0 + 5, mapcxy, static_cast<size_t>(nsea), s);
    int* d_th2 = st.in(k0 + 6, mapth2, nth2, s);
    int* d_wn2 = st.in(k0 + 7, mapwn2, nwn2, s);
    Map3Work& w = map3_work();
    launch_map3(Map3Grid{nx, ny, nsea, nk, nth, gtype}, d_sta, d_sf, d_x2, d_y2, d_axy, d_cxy,
                d_th2, d_wn2, w, s);
    auto out = [&](int* h, const int* d, size_t n) {
      if (n) WWB_CHECK(cudaMemcpyAsync(h, d, n * sizeof(int), cudaMemcpyDeviceToHost, s));
    };
    if (gtype < 3) {
      out(mapx2, d_x2, nxy);
      out(mapy2, d_y2, nxy);
      out(mapaxy, d_axy, nxy);
      out(mapcxy, d_cxy, static_cast<size_t>(nsea));
      out(counts, w.counts, 8);
    }
    out(mapth2, d_th2, nth2);
    out(mapwn2, d_wn2, nwn2);
    WWB_CHECK(cudaStreamSynchronize(s));
    g_prop3.ok();
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_map3_device(int nx, int ny, int nsea, int nk, int nth, int gtype, const int* mapsta,
                   const int* mapsf, int* mapx2, int* mapy2, int* mapaxy, int* mapcxy,
                   int* mapth2, int* mapwn2, int* counts, void* stream) {
  return guarded([&] {
    if (const int rc = map3_check(nx, ny, nsea, nk, nth, mapsta, mapsf, mapx2, mapy2, mapaxy,
                                  mapcxy, mapth2, mapwn2, counts, false);
        rc != WW_KOKKOS_OK)
      return rc;
    if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Map3Work& w = map3_work();
    launch_map3(Map3Grid{nx, ny, nsea, nk, nth, gtype}, mapsta, mapsf, mapx2, mapy2, mapaxy,
                mapcxy, mapth2, mapwn2, w, s);
    if (gtype < 3) {
      WWB_CHECK(cudaMemcpyAsync(counts, w.counts, 8 * sizeof(int), cudaMemcpyDeviceToHost, s));
      WWB_CHECK(cudaStreamSynchronize(s));
    }
    g_prop3.ok();
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_mapt(int nx, int ny, int nsea, const int* mapsf, const float* atrnx, const float* atrny,
            int* maptrn) {
  return guarded([&] {
    if (nx < 1 || ny < 1 || nsea < 0 || (nsea > 0 && (!mapsf || !atrnx || !atrny || !maptrn)))
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_mapt: bad sizes or null pointer");
    const long long nxy = static_cast<long long>(nx) * ny;
    for (int i = 0; i < nsea; ++i)
      if (mapsf[2 * nsea + i] < 1 || mapsf[2 * nsea + i] > nxy)
        return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_mapt: MAPSF(:,3) outside the grid");
    if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
    if (nsea == 0) {
      g_prop3.ok();
      return static_cast<int>(WW_KOKKOS_OK);
    }
    Staging& st = staging();
    cudaStream_t s = runtime().stream;
    constexpr int k0 = 90;
    const int* d_sf = st.in(k0, mapsf, 3 * static_cast<size_t>(nsea), s);
    const float* d_x = st.in(k0 + 1, atrnx, 3 * static_cast<size_t>(nxy), s);
    const float* d_y = st.in(k0 + 2, atrny, 3 * static_cast<size_t>(nxy), s);
    int* d_t = st.in(k0 + 3, maptrn, static_cast<size_t>(nxy), s);
    launch_mapt(nsea, static_cast<int>(nxy), d_sf, d_x, d_y, d_t, s);
    WWB_CHECK(cudaMemcpyAsync(maptrn, d_t, sizeof(int) * nxy, cudaMemcpyDeviceToHost, s));
    WWB_CHECK(cudaStreamSynchronize(s));
    g_prop3.ok();
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_utrn(int nx, int ny, int nsea, int trflag, float fice0, float ficen, float ficel,
            float ffacberg, int flagll, float trny_before, const float* trnx, const float* trny,
            const int* mapsf, const int* mapsta, const float* hpfac, const float* hqfac,
            const float* ice, const float* berg, float* atrnx, float* atrny) {
  return guarded([&] {
    if (nx < 1 || ny < 1 || nsea < 0 || static_cast<long long>(nx) * ny > (1ll << 31) - 1 ||
        !atrnx || !atrny || (nsea > 0 && (!mapsf || !mapsta || !trnx || !trny)))
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_utrn: bad sizes or null pointer");
    const UtrnGrid g{nx, ny, nsea, trflag, fice0, ficen, ficel, ffacberg, flagll ? 1 : 0,
                     trny_before};
    const bool ice_on = trflag != 0 && utrn_needs_ice(g);
    if (ice_on && nsea > 0 && (!hpfac || !hqfac || !ice || !berg))
      return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_utrn: ice arrays missing");
    for (int i = 0; i < nsea; ++i) {
      const int ix = mapsf[i], iy = mapsf[nsea + i], ixy = mapsf[2 * nsea + i];
      if (ix < 1 || ix > nx || iy < 1 || iy > ny || ixy != (ix - 1) * ny + iy)
        return fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_utrn: MAPSF is not a map of cells of the grid");
    }
    if (!runtime().ready) return fail(WW_KOKKOS_ERR_NOT_INITIALISED, "before ww_kokkos_init");
    timers::Region t_call("utrn.call");
    Staging& st = staging();
    cudaStream_t s = runtime().stream;
    const size_t nxy = static_cast<size_t>(nx) * ny, ns = static_cast<size_t>(nsea);
    constexpr int k0 = 100;
    const int* d_sf = nsea ? st.in(k0, mapsf, 3 * ns, s) : nullptr;
    const int* d_sta = nsea ? st.in(k0 + 1, mapsta, nxy, s) : nullptr;
    const float* d_tx = nsea ? st.in(k0 + 2, trnx, nxy, s) : nullptr;
    const float* d_ty = nsea ? st.in(k0 + 3, trny, nxy, s) : nullptr;
    const bool ice_arrays = ice_on && nsea > 0;
    const float* d_hp = ice_arrays ? st.in(k0 + 4, hpfac, nxy, s) : nullptr;
    const float* d_hq = ice_arrays ? st.in(k0 + 5, hqfac, nxy, s) : nullptr;
    const float* d_ice = ice_arrays ? st.in(k0 + 6, ice, ns + 1, s) : nullptr;
    const float* d_berg = ice_arrays ? st.in(k0 + 7, berg, ns, s) : nullptr;
    float* d_ax = static_cast<float*>(st.get(k0 + 8, 3 * nxy * sizeof(float)));
    float* d_ay = static_cast<float*>(st.get(k0 + 9, 3 * nxy * sizeof(float)));
    float* d_tri = ice_on ? static_cast<float*>(st.get(k0 + 10, 2 * nxy * sizeof(float))) : nullptr;
    launch_utrn(g, d_sf, d_sta, d_tx, d_ty, d_hp, d_hq, d_ice, d_berg, d_ax, d_ay, d_tri,
                d_tri ? d_tri + nxy : nullptr, s);
    WWB_CHECK(cudaMemcpyAsync(atrnx, d_ax, 3 * nxy * sizeof(float), cudaMemcpyDeviceToHost, s));
    WWB_CHECK(cudaMemcpyAsync(atrny, d_ay, 3 * nxy * sizeof(float), cudaMemcpyDeviceToHost, s));
    WWB_CHECK(cudaStreamSynchronize(s));
    g_prop3.ok();
    return static_cast<int>(WW_KOKKOS_OK);
  });
}

int ww_prop3_last_error(void) { return g_prop3.get(); }

}  // extern "C"
