// oracle/ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Flat extern "C" access to the INSNL1 tables of the reference's own C++
// (ww::snl1::make_tables, ww3-gpu kokkos/src/ww_kokkos/snl1_tables.cpp:82-329), compiled from
// the reference's sources by oracle/Makefile into oracle/_ref/libref_ww3.so. The reference's
// W3SNL1 itself is reached through its own C ABI in the same library (ww_kokkos_init,
// ww_snl1_init, ww_snl1: kokkos/src/fortran_iface/snl1_shim.cpp), so no driver is needed for
// it, nor for W3KTP3/W3XYP3 (ww_ktp3_batch, ww_xyp3_batch: prop3_shim.cpp) and the resident VA
// (ww_va_*: resident_shim.cpp). Used by the tests and by bench.py's reference arm only.
#include <Kokkos_Core.hpp>
#include <vector>

#include "ww_kokkos/snl1_config.hpp"
#include "ww_kokkos/snl1_tables.hpp"

extern "C" int ref_snl1_tables(int nk, int nth, float xfr, float dth, float lam, float snlc1,
                               float kdcon, float kdmn, float snls1, float snls2, float snls3,
                               float fachfe, const float* sig, int* scal, float* wts,
                               int* ipim, int* ic, float* af11, int* halo) {
  const ww::snl1::Config c{nk, nth, xfr, dth, lam, snlc1, kdcon, kdmn, snls1, snls2, snls3, fachfe};
  ww::snl1::HostRealView1D h_sig("sig", nk);
  for (int k = 0; k < nk; ++k) h_sig(k) = sig[k];
  const ww::snl1::Tables t = ww::snl1::make_tables(c, h_sig);
  scal[0] = t.nfr;
  scal[1] = t.nfrhgh;
  scal[2] = t.nfrchg;
  scal[3] = t.nspecx;
  scal[4] = t.nspecy;
  wts[0] = t.dal1;
  wts[1] = t.dal2;
  wts[2] = t.dal3;
  for (int j = 0; j < 8; ++j) {
    wts[3 + j] = t.awg[j];
    wts[11 + j] = t.swg[j];
  }
  if (halo) *halo = t.halo;
  if (ipim) {
    for (int half = 0; half < 2; ++half)
      for (int j = 0; j < 4; ++j)
        for (int i = 0; i < t.nspecx; ++i) {
          ipim[(half * 8 + j) * t.nspecx + i] = t.ip[half][j](i);
          ipim[(half * 8 + 4 + j) * t.nspecx + i] = t.im[half][j](i);
        }
  }
  if (ic) {
    for (int j = 0; j < 8; ++j)
      for (int col = 0; col < 2; ++col)
        for (int i = 0; i < t.nspec; ++i) ic[(col * 8 + j) * t.nspec + i] = t.ic[j][col](i);
  }
  if (af11)
    for (int i = 0; i < t.nspecx; ++i) af11[i] = t.af11(i);
  return 0;
}

// prop3_shim.cpp's exit report names the unstructured-grid shim's counter, which this build
// leaves out (that propagation scheme is not on the path); an empty report stands in for it.
extern "C" void ww_xypug_report(void) {}

// W3MAP3 of the reference (kokkos/src/ww_kokkos/prop_map3.hpp:65-340), to build the PR3 maps of
// synthetic grids for the tests: mapsta (NY*NX), mapsf (NSEA,3) column-major in; mapx2, mapy2,
// mapaxy (NY*NX), mapcxy (NSEA), mapth2 ((NK+2)*NTH, zeroed), mapwn2 (NK*NTH+NTH) and
// counts[8] = NMX0, NMX1, NMX2, NMY0, NMY1, NMY2, NACT, NCENT out.
#include "ww_kokkos/prop_map3.hpp"

extern "C" int ref_w3map3(int nx, int ny, int nsea, int nk, int nth, const int* mapsta,
                          const int* mapsf, int* mapx2, int* mapy2, int* mapaxy, int* mapcxy,
                          int* mapth2, int* mapwn2, int* counts) {
  using namespace ww::prop;
  Map3Scalars s{nx, ny, nsea, nk, nth, 1};
  using V = Map3Views<Kokkos::HostSpace>;
  V v;
  v.mapsta = V::I1(mapsta, static_cast<size_t>(nx) * ny);
  v.mapsf = V::I2(mapsf, static_cast<size_t>(nsea), 3);
  v.mapx2 = V::W1(mapx2, static_cast<size_t>(nx) * ny);
  v.mapy2 = V::W1(mapy2, static_cast<size_t>(nx) * ny);
  v.mapaxy = V::W1(mapaxy, static_cast<size_t>(nx) * ny);
  v.mapcxy = V::W1(mapcxy, static_cast<size_t>(nsea));
  v.mapth2 = V::W1(mapth2, static_cast<size_t>(nk + 2) * nth);
  v.mapwn2 = V::W1(mapwn2, static_cast<size_t>(nk) * nth + nth);
  v.counts = V::W1(counts, 8);
  Map3Counts c{};
  w3map3(Kokkos::DefaultHostExecutionSpace(), s, v, c);
  return 0;
}

// W3MAPT of the reference (kokkos/src/ww_kokkos/prop_mapt.hpp:55-79): MAPTRN of the NSEA sea
// cells from ATRNX/ATRNY (NY*NX, -1:1), column-major.
#include "ww_kokkos/prop_mapt.hpp"

extern "C" int ref_w3mapt(int nx, int ny, int nsea, const int* mapsf, const float* atrnx,
                          const float* atrny, int* maptrn) {
  using namespace ww::prop;
  using H = Kokkos::HostSpace;
  const size_t nxy = static_cast<size_t>(nx) * ny;
  Kokkos::View<const int**, Kokkos::LayoutLeft, H> sf(mapsf, static_cast<size_t>(nsea), 3);
  Kokkos::View<const float**, Kokkos::LayoutLeft, H> ax(atrnx, nxy, 3), ay(atrny, nxy, 3);
  Kokkos::View<int*, Kokkos::LayoutLeft, H> t(maptrn, nxy);
  w3mapt(Kokkos::DefaultHostExecutionSpace(), nsea, sf, ax, ay, t);
  return 0;
}

// W3UTRN of the reference (kokkos/src/ww_kokkos/updt_utrn.hpp:302-362): ATRNX/ATRNY
// (NY*NX, 3) from TRNX/TRNY, ICE (0:NSEA), BERG (NSEA), MAPSF (NSEA,3), MAPSTA/HPFAC/HQFAC (NY,NX).
#include "ww_kokkos/updt_utrn.hpp"

extern "C" int ref_w3utrn(int nx, int ny, int nsea, int trflag, float fice0, float ficen,
                          float ficel, float ffacberg, int flagll, float trny_before,
                          const float* trnx, const float* trny, const int* mapsf,
                          const int* mapsta, const float* hpfac, const float* hqfac,
                          const float* ice, const float* berg, float* atrnx, float* atrny) {
  using namespace ww::updt;
  using V = UtrnViews<Kokkos::HostSpace>;
  const size_t nxy = static_cast<size_t>(nx) * ny;
  UtrnScalars s{};
  s.nx = nx;
  s.ny = ny;
  s.nsea = nsea;
  s.trflag = trflag;
  s.fice0 = fice0;
  s.ficen = ficen;
  s.ficel = ficel;
  s.ffacberg = ffacberg;
  s.flagll = flagll != 0;
  s.trny_before = trny_before;
  std::vector<float> tri(2 * nxy, 0.0f);
  V v;
  v.trnx = V::R1(trnx, nxy);
  v.trny = V::R1(trny, nxy);
  v.ice = V::R1(ice, static_cast<size_t>(nsea) + 1);
  v.berg = V::R1(berg, static_cast<size_t>(nsea > 0 ? nsea : 1));
  v.mapsf = V::I2(mapsf, static_cast<size_t>(nsea), 3);
  v.mapsta = V::I2(mapsta, static_cast<size_t>(ny), static_cast<size_t>(nx));
  v.hpfac = V::R2(hpfac, static_cast<size_t>(ny), static_cast<size_t>(nx));
  v.hqfac = V::R2(hqfac, static_cast<size_t>(ny), static_cast<size_t>(nx));
  v.atrnx = V::W2(atrnx, nxy, 3);
  v.atrny = V::W2(atrny, nxy, 3);
  v.trix = V::W1(tri.data(), nxy);
  v.triy = V::W1(tri.data() + nxy, nxy);
  w3utrn(Kokkos::DefaultHostExecutionSpace(), s, v);
  return 0;
}

// INSIN4(FLTABS=.TRUE.) of the reference (kokkos/src/ww_kokkos/st4_insin4.cpp, st4_tabu_*.cpp),
// to build the ST4 tables of synthetic grids for the tests. rpar/ipar are the ST4 packets
// (st4_params.hpp:79-154); sig, dsip are SIG(0:MK+1), DSIP(0:MK+1). Out, column-major with the
// shapes of st4_arrays.hpp:93-114 (allocate_tables); th = TH(1:MTH), ecos = ECOS(1:MSPEC+MTH): satweights, satindices (2*(MTH/2-1)+1, MTH),
// iktab (MK, NDTAB), dcki, qbi (NKHS, NKD), cumulw (MSPEC, MSPEC), taut (ITAUMAX+1, JUMAX+1),
// tauhft (IUSTAR+1, IALPHA+1), tauhft2 (IUSTAR+1, IALPHA+1, ILEVTAIL+1) (may be null when not
// allocated), del[5] = DELUST, DELALP, DELTAUW, DELU, DELTAIL.
#include "ww_kokkos/st4_tables_build.hpp"

extern "C" int ref_st4_tables(const float* rpar, const int* ipar, const float* sig,
                              const float* dsip, const float* th, const float* ecos,
                              float* satweights, int* satindices, int* iktab,
                              float* dcki, float* qbi, float* cumulw, float* taut, float* tauhft,
                              float* tauhft2, float* del) {
  using namespace ww::st4;
  Params p = unpack(rpar, ipar);
  HostArrays a;
  a.sig = HostArrays::V1<float>("sig", p.mk + 2);
  a.dsip = HostArrays::V1<float>("dsip", p.mk + 2);
  for (int i = 0; i < p.mk + 2; ++i) {
    a.sig(i) = sig[i];
    a.dsip(i) = dsip[i];
  }
  a.th = HostArrays::V1<float>("th", p.mth);
  for (int i = 0; i < p.mth; ++i) a.th(i) = th[i];
  a.ecos = HostArrays::V1<float>("ecos", p.mspec + p.mth);
  for (int i = 0; i < p.mspec + p.mth; ++i) a.ecos(i) = ecos[i];
  allocate_tables(p, a);
  insin4(p, true, a);
  auto out = [](const auto& v, auto* dst) {
    if (dst && v.data()) std::memcpy(dst, v.data(), sizeof(*dst) * v.size());
  };
  out(a.satweights, satweights);
  out(a.satindices, satindices);
  out(a.iktab, iktab);
  out(a.dcki, dcki);
  out(a.qbi, qbi);
  out(a.cumulw, cumulw);
  out(a.taut, taut);
  out(a.tauhft, tauhft);
  out(a.tauhft2, tauhft2);
  del[0] = p.delust;
  del[1] = p.delalp;
  del[2] = p.deltauw;
  del[3] = p.delu;
  del[4] = p.deltail;
  return 0;
}

// W3CFLXY of the reference (kokkos/src/ww_kokkos/prop_cflxy.hpp:61-135) for ISEA = 1..NSEA, as
// its W3WAVE driver calls it (wave_w3wave.hpp:563-572; mgp selects the W3_MGP form): mapsf
// (NSEA,3) column-major, clats (0:NSEA), ecos/esin (NTH), dpdx..dqdy (NY,NX), cg (0:NK+1,0:NSEA),
// cx/cy (0:NSEA) in; cflxymax (NSEA) out.
#include "ww_kokkos/prop_cflxy.hpp"

extern "C" int ref_w3cflxy(int nsea, int nx, int ny, int nk, int nth, int flcur, int mgp,
                           float dtg, float vgx, float vgy, const int* mapsf, const float* clats,
                           const float* ecos, const float* esin, const float* dpdx,
                           const float* dpdy, const float* dqdx, const float* dqdy,
                           const float* cg, const float* cx, const float* cy, float* cflxymax) {
  using namespace ww::prop;
  Params p{};
  p.nx = nx;
  p.ny = ny;
  p.nsea = nsea;
  p.nk = nk;
  p.nth = nth;
  p.nspec = nk * nth;
  p.flcur = flcur;
  Grid g{};
  g.mapsf = mapsf;
  g.clats = clats;
  g.ecos = ecos;
  g.esin = esin;
  g.dpdx = dpdx;
  g.dpdy = dpdy;
  g.dqdx = dqdx;
  g.dqdy = dqdy;
  Step s{};
  s.cg = cg;
  s.cx = cx;
  s.cy = cy;
  for (int isea = 1; isea <= nsea; ++isea) {
    if (mgp)
      w3cflxy<true>(isea, dtg, nullptr, nullptr, cflxymax[isea - 1], vgx, vgy, p, g, s);
    else
      w3cflxy<false>(isea, dtg, nullptr, nullptr, cflxymax[isea - 1], vgx, vgy, p, g, s);
  }
  return 0;
}

// The GQM table builders of the reference (kokkos/src/ww_kokkos/snl1_couple.hpp:37-88,
// snl1_gauleg.hpp:28-61, snl1_f1f1f1.hpp:37-145), header-only, for the tests: COUPLE over n
// quadruplets k (8, n) column-major; GAULEG; F1F1F1 (returns its diagnostic bits).
#include "ww_kokkos/snl1_couple.hpp"
#include "ww_kokkos/snl1_f1f1f1.hpp"
#include "ww_kokkos/snl1_gauleg.hpp"

extern "C" int ref_gqm_couple(int n, const double* k, double* coef, int* diag) {
  for (int i = 0; i < n; ++i) {
    const double* c = k + 8 * static_cast<size_t>(i);
    int d = 0;
    coef[i] = ww::snl1::couple(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], d);
    diag[i] = d;
  }
  return 0;
}

extern "C" int ref_gqm_gauleg(int npoin, double* w_leg, double* x_leg) {
  ww::snl1::gauleg(w_leg, x_leg, npoin);
  return 0;
}

extern "C" int ref_gqm_f1f1f1(int* nf1, int iq_om1, double* f1sf) {
  return ww::snl1::f1f1f1(f1sf, *nf1, iq_om1);
}
