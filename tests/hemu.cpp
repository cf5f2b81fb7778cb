// tests/hemu.cpp -- the host build of the ST4 / W3SRCE kernels' source (csrc/st4_point.cuh,
// csrc/srce_point.cuh), for the CPU tests: the same phases the CUDA kernels run, executed by one
// host "thread" per point, behind entry points that take the reference's C ABI arguments (minus
// igrid: one grid). The CPU tests compare these with the reference's own build (oracle/_ref), so
// the kernels' arithmetic is checked without a GPU; the GPU tests then compare the CUDA library
// with the same reference. Compiled by tests/conftest.py with -ffp-contract=off.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "snl1_tables.hpp"
#include "srce_point.cuh"
#include "st4_registry.hpp"

using namespace wwb;

namespace {
st4::GridReg g_grid;
st4::ModuleReg g_mod;
std::vector<float> g_satw_t;
std::vector<int> g_sati_t;
std::vector<float> g_cumulw_t;
pt::Fields g_fields{};
st4::Params g_p{};
bool g_ready = false;

Snl1Config g_ncfg{};
Snl1Tables g_ntab;
std::vector<float> g_nsig;
Snl1Dev g_ndev{};

srce::Params g_sp{};
std::vector<float> g_ssig, g_sdden, g_secos, g_sesin;
std::vector<int> g_smapwn;
pt::SrceGrid g_sgrid{};

const float* fp(const st4::Reg& r) { return r.f.empty() ? nullptr : r.f.data(); }
const int* ip(const st4::Reg& r) { return r.i.empty() ? nullptr : r.i.data(); }
}  // namespace

extern "C" {

int hemu_st4_init(const float* rpar, int nrpar, const int* ipar, int nipar) {
  if (nrpar != st4::NRPAR || nipar != st4::NIPAR) return 2;
  g_grid = st4::GridReg{};
  g_grid.p = st4::unpack(rpar, ipar);
  g_grid.configured = true;
  g_mod.delust = g_grid.p.delust;
  g_mod.delalp = g_grid.p.delalp;
  g_mod.deltauw = g_grid.p.deltauw;
  g_mod.delu = g_grid.p.delu;
  g_mod.deltail = g_grid.p.deltail;
  g_mod.delab = g_grid.p.delab;
  g_ready = false;
  return 0;
}

int hemu_st4_set_real(int id, const float* data, int rank, const int* lb, const int* ext) {
  std::string why;
  return st4::reg_set(g_grid, g_mod, id, data, false, rank, lb, ext, why);
}

int hemu_st4_set_int(int id, const int* data, int rank, const int* lb, const int* ext) {
  std::string why;
  return st4::reg_set(g_grid, g_mod, id, data, true, rank, lb, ext, why);
}

int hemu_st4_commit(void) {
  std::string why;
  if (!st4::reg_check(g_grid, g_mod, why)) {
    std::fprintf(stderr, "hemu_st4_commit: %s\n", why.c_str());
    return 6;
  }
  st4::transpose_sat(g_grid, g_satw_t, g_sati_t);
  st4::transpose_cumulw(g_grid, g_cumulw_t);
  const auto& a = g_grid.a;
  const auto& m = g_mod.a;
  st4::FieldPtrs q{fp(a[st4::A_SIG]), fp(a[st4::A_SIG2]), fp(a[st4::A_DSIP]),
                   fp(a[st4::A_DDEN]), fp(a[st4::A_DDEN2]), fp(a[st4::A_ESIN]),
                   fp(a[st4::A_ECOS]), fp(a[st4::A_TH]), g_satw_t.data(),
                   g_cumulw_t.data(), fp(a[st4::A_DCKI]), fp(a[st4::A_QBI]),
                   fp(m[st4::A_TAUT]), fp(m[st4::A_TAUHFT]), fp(m[st4::A_TAUHFT2]),
                   fp(m[st4::A_FWTABLE]), g_sati_t.data(), ip(a[st4::A_IKTAB])};
  g_fields = st4::make_fields(g_grid, q);
  g_p = st4::current_params(g_grid, g_mod);
  g_ready = true;
  return 0;
}

void hemu_sds4(int npts, const float* a, const float* k, const float* cg, const float* ustar,
               const float* usdir, const float* depth, const float* dair, const float* dlwmean,
               int flogrd57, int flogrd58, float* srhs, float* ddiag, float* brlambda,
               float* whitecap) {
  const st4::Params& p = g_p;
  std::vector<float> w(pt::sds4_work_reals(p)), w2(pt::sds4_work2_reals(p));
  std::vector<int> iw(pt::sds4_work_ints(p));
  pt::Sds4Sh sh{};
  const pt::Cta cta{0, 1};
  for (int n = 0; n < npts; ++n) {
    const size_t os = static_cast<size_t>(n) * p.nspec, ok = static_cast<size_t>(n) * p.nk;
    pt::sds4(cta, p, g_fields, a + os, k + ok, cg + ok, ustar[n], usdir[n], depth[n], dair[n],
             dlwmean[n], flogrd57, flogrd58, srhs + os, ddiag + os, brlambda + os,
             whitecap + 4 * static_cast<size_t>(n), w.data(), w2.data(), iw.data(), sh);
  }
}

void hemu_sin4(int npts, const float* a, const float* cg, const float* k, const float* u,
               const float* ustar, const float* drat, const float* as, const float* usdir,
               const float* z0, const float* cd, float* tauwx, float* tauwy, float* tauwnx,
               float* tauwny, float* s, float* d, int* llws) {
  (void)cd;
  const st4::Params& p = g_p;
  std::vector<float> dstab(3 * p.nspec), eb(pt::sin4_nk_work(p));
  static pt::Sin4Sh sh;
  const pt::Cta cta{0, 1};
  for (int n = 0; n < npts; ++n) {
    const size_t os = static_cast<size_t>(n) * p.nspec, ok = static_cast<size_t>(n) * p.nk;
    pt::sin4(cta, p, g_fields, a + os, cg + ok, k + os, p.nth, u[n], ustar[n], drat[n], as[n],
             usdir[n], z0[n], tauwx + n, tauwy + n, tauwnx + n, tauwny + n, s + os, d + os,
             llws + os, dstab.data(), eb.data(), sh);
  }
}

void hemu_spr4(int npts, const float* a, const float* cg, const float* wn, const float* u,
               const float* udir, const float* tauwx, const float* tauwy, const int* llws,
               float* ustar, float* usdir, float* emean, float* fmean, float* fmean1,
               float* wnmean, float* amax, float* cd, float* z0, float* charn, float* fmeanws,
               float* dlwmean) {
  const st4::Params& p = g_p;
  std::vector<float> w(pt::spr4_work_reals(p)), terms(pt::spr4_terms_reals(p));
  const pt::Cta cta{0, 1};
  for (int n = 0; n < npts; ++n) {
    const size_t os = static_cast<size_t>(n) * p.nspec, ok = static_cast<size_t>(n) * p.nk;
    pt::Spr4Out o{ustar[n], usdir[n], emean[n], fmean[n], fmean1[n], wnmean[n],
                  amax[n],  cd[n],    z0[n],    charn[n], fmeanws[n], dlwmean[n]};
    pt::spr4(cta, p, g_fields, a + os, cg + ok, wn + ok, u[n], udir[n], tauwx[n], tauwy[n],
             llws + os, o, w.data(), terms.data());
    ustar[n] = o.ustar;
    usdir[n] = o.usdir;
    emean[n] = o.emean;
    fmean[n] = o.fmean;
    fmean1[n] = o.fmean1;
    wnmean[n] = o.wnmean;
    amax[n] = o.amax;
    cd[n] = o.cd;
    z0[n] = o.z0;
    charn[n] = o.charn;
    fmeanws[n] = o.fmeanws;
    dlwmean[n] = o.dlwmean;
  }
}

int hemu_snl1_init(int nk, int nth, float xfr, float dth, float lam, float snlc1, float kdcon,
                   float kdmn, float snls1, float snls2, float snls3, float fachfe,
                   const float* sig) {
  g_ncfg = Snl1Config{nk, nth, xfr, dth, lam, snlc1, kdcon, kdmn, snls1, snls2, snls3, fachfe};
  g_ntab = Snl1Tables{};
  if (!build_snl1_tables(g_ncfg, sig, g_ntab) || !g_ntab.rowshift) return 2;
  g_nsig.assign(sig, sig + nk);
  Snl1Dev& p = g_ndev;
  p = Snl1Dev{};
  p.nk = nk;
  p.nth = nth;
  p.nfr = g_ntab.nfr;
  p.nfrhgh = g_ntab.nfrhgh;
  p.nfrchg = g_ntab.nfrchg;
  p.nspec = g_ntab.nspec;
  p.nspecx = g_ntab.nspecx;
  p.dal1 = g_ntab.dal1;
  p.dal2 = g_ntab.dal2;
  p.dal3 = g_ntab.dal3;
  for (int j = 0; j < 8; ++j) {
    p.awg[j] = g_ntab.awg[j];
    p.swg[j] = g_ntab.swg[j];
    p.shift[j] = g_ntab.shift[j];
  }
  p.ifrp = g_ntab.ifrp;
  p.ifrm = g_ntab.ifrm;
  p.snlc1 = snlc1;
  p.kdcon = kdcon;
  p.kdmn = kdmn;
  p.snls1 = snls1;
  p.snls2 = snls2;
  p.snls3 = snls3;
  p.fachfe = fachfe;
  p.ifrow = g_ntab.ifrow.data();
  p.af11_row = g_ntab.af11_row.data();
  p.sig = g_nsig.data();
  return 0;
}

int hemu_srce_init(const float* rpar, int nrpar, const int* ipar, int nipar, const float* sig,
                   const float* dden, const float* ecos, const float* esin, const int* mapwn) {
  if (nrpar != srce::NRPAR || nipar != srce::NIPAR) return 2;
  g_sp = srce::unpack(rpar, ipar);
  const int nk = g_sp.nk, ns = g_sp.nspec;
  g_ssig.assign(sig, sig + nk);
  g_sdden.assign(dden, dden + nk);
  g_secos.assign(ecos, ecos + ns);
  g_sesin.assign(esin, esin + ns);
  g_smapwn.assign(mapwn, mapwn + ns);
  g_sgrid = pt::SrceGrid{g_ssig.data(), g_sdden.data(), g_secos.data(), g_sesin.data(),
                         g_smapwn.data()};
  return 0;
}

/// ww_srce_batch without igrid: points one after the other.
void hemu_srce_batch(int it, int inflags24, int flogrd57, int flogrd58, float dtg, int npts,
                     float* spec, const float* wn1, const float* cg1, const float* pin,
                     float* psc, float* whitecap, float* taubbl, float* tauice, int* shave) {
  const pt::SrceLayout L = pt::srce_layout(g_p, g_ndev);
  std::vector<float> w(L.total_s + 4), gw(L.total_g + 4);
  static pt::SrceSh sh;
  const pt::Cta cta{0, 1};
  const int ns = g_sp.nspec, nk = g_sp.nk;
  for (int n = 0; n < npts; ++n) {
    float* const sp = spec + static_cast<size_t>(n) * ns;
    const float* const pi = pin + static_cast<size_t>(n) * srce::NPIN;
    float* const ps = psc + static_cast<size_t>(n) * srce::NPSC;
    std::memcpy(w.data() + L.spec, sp, sizeof(float) * ns);
    std::memcpy(w.data() + L.wn1, wn1 + static_cast<size_t>(n) * nk, sizeof(float) * nk);
    std::memcpy(w.data() + L.cg1, cg1 + static_cast<size_t>(n) * nk, sizeof(float) * nk);
    pt::srce_psc_in(sh, ps, whitecap + 4 * static_cast<size_t>(n),
                    taubbl + 2 * static_cast<size_t>(n), tauice + 2 * static_cast<size_t>(n));
    pt::SrceCtx x{&g_sp, &g_sgrid, &g_p, &g_fields, &g_ndev,
                  pt::srce_in(it, inflags24, flogrd57, flogrd58, dtg, pi), w.data(), gw.data(),
                  &L, &sh};
    pt::srce_point(cta, x);
    std::memcpy(sp, w.data() + L.spec, sizeof(float) * ns);
    pt::srce_psc_out(sh, ps, whitecap + 4 * static_cast<size_t>(n),
                     taubbl + 2 * static_cast<size_t>(n), tauice + 2 * static_cast<size_t>(n),
                     shave + n);
  }
}

}  // extern "C"
