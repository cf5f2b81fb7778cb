// ww3-gpu_b200/csrc/outg_kernel.cu
// W3OUTG on sm_100a (see outg_kernel.cuh): one thread per sea point reads its column of the
// resident VA and forms every integral in the reference's statement order.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/iogo_w3outg.hpp:198-598 (w3outg_point: sections 2-4 and
// the space-time extremes of w3iogomd.F90:1201-2380), :603-690 (w3outg_part_point, section 6),
// :693-713 (the whole-array assignments of section 1). The sums over ITH and IK of a point are
// sequential in the reference, so a point is one thread: no reduction is reordered. MAX/MIN keep
// the object's operand order per site (gt_sel / lt_sel), the folded PARAMETERs their float bits,
// and the libm calls are the glibc-equal device functions; the THMP sine and cosine, which the
// reference's host object takes from libmvec's 4-lane entries for most points, are the scalar
// sinf/cosf here (the bits the reference gives with those entries bound to scalar calls).
#include "outg_kernel.cuh"

#include "libm_dev.cuh"
#include "wwb_common.hpp"

namespace wwb {
namespace {

constexpr float kPi = static_cast<float>(3.141592653589793);
constexpr float kTpi = 2.0f * kPi;
constexpr float kTpiInv = 1.0f / kTpi;
constexpr float kGrav = 9.806f;
constexpr float kDwat = 1000.0f;
constexpr float kRade = 180.0f / kPi;
constexpr float kDera = kPi / 180.0f;
constexpr float kTpi2 = kTpi * kTpi;
constexpr float kGrav2 = kGrav * kGrav;
constexpr float kRadeHalf = kRade * 0.5f;
constexpr float kRade001 = 0.01f * kRade;
constexpr float kDwatGrav = kDwat * kGrav;
constexpr float kSqrtTpi = 0x1.40d932p+1f;  // SQRT(TPI) as folded
constexpr float kSqrt6 = 0x1.3988e2p+1f;    // SQRT(6.)
constexpr float kPiSqrt6 = kPi / kSqrt6;
static_assert(kTpi2 == 3.9478420257568359375e+1f, "TPI**2");
static_assert(kGrav2 == 9.615763092041015625e+1f, "GRAV**2");
static_assert(kRade == 5.72957763671875e+1f && kRadeHalf == 2.864788818359375e+1f, "RADE");
static_assert(kRade001 == 5.729577541351318359375e-1f, "0.01*RADE");
static_assert(kDwatGrav == 9.806e+3f, "DWAT*GRAV");
static_assert(kPiSqrt6 == 1.28254985809326171875f, "PI/SQRT(6.)");
static_assert(kDera == 1.745329238474369049072265625e-2f, "DERA");

__device__ __forceinline__ float gt_sel(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float lt_sel(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float cosf_(float x) {
  float s, c;
  dm::sincosf(x, &s, &c);
  return c;
}

/// A result stored as the reference's x86-64 object stores it: every invalid operation there
/// (the square root or logarithm of a negative number, 0/0) gives the default NaN 0xFFC00000,
/// which the later operations carry unchanged, where the device's canonical NaN is 0x7FFFFFFF.
/// The inputs are finite, so each NaN of a field is that default NaN.
__device__ __forceinline__ void put(float* f, size_t i, float v) {
  f[i] = (v == v) ? v : __int_as_float(static_cast<int>(0xffc00000u));
}

#define F1(k) a.f[k][j0]

__global__ void outg_init_kernel(OutgArgs a) {
  const float z = 0.0f, undef = a.undef;
  for (int j0 = blockIdx.x * blockDim.x + threadIdx.x; j0 < a.nfld; j0 += gridDim.x * blockDim.x) {
    F1(OG_ABA) = z; F1(OG_ABD) = z; F1(OG_UBA) = z; F1(OG_UBD) = z;
    F1(OG_SXX) = z; F1(OG_SYY) = z; F1(OG_SXY) = z;
    F1(OG_USSX) = z; F1(OG_USSY) = z; F1(OG_TUSX) = z; F1(OG_TUSY) = z;
    F1(OG_MSSX) = z; F1(OG_MSSY) = z; F1(OG_MSSD) = z; F1(OG_MSCX) = z; F1(OG_MSCY) = z;
    F1(OG_MSCD) = z; F1(OG_PRMS) = z; F1(OG_TPMS) = z; F1(OG_BHD) = z;
    F1(OG_HS) = undef; F1(OG_WLM) = undef; F1(OG_T0M1) = undef; F1(OG_T01) = undef;
    F1(OG_T02) = undef; F1(OG_FP0) = undef; F1(OG_THM) = undef; F1(OG_THS) = undef;
    F1(OG_THP0) = undef; F1(OG_HSIG) = undef; F1(OG_QKK) = undef; F1(OG_STMAXE) = undef;
    F1(OG_STMAXD) = undef; F1(OG_HCMAXE) = undef; F1(OG_HMAXE) = undef; F1(OG_HCMAXD) = undef;
    F1(OG_HMAXD) = undef; F1(OG_QP) = undef; F1(OG_WBT) = undef;
  }
}

__global__ void __launch_bounds__(128) outg_point_kernel(OutgArgs a) {
  const int jsea = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (jsea > a.nseal) return;
  const float zero = 0.0f, half = 0.5f, one = 1.0f, two = 2.0f, k1em7 = 1.E-7f;
  const int nk = a.nk, nth = a.nth, nk2 = nk + 2;
  const int j0 = jsea - 1;
  const int isea = jsea;  // W3_SHRD: ISEA = JSEA
  const int ix = a.mapsf[isea - 1], iy = a.mapsf[a.nsea + isea - 1];
  // A MAPSF cell outside the grid (only a device caller can pass one unchecked) reads as land.
  const bool in_grid = ix >= 1 && ix <= a.nx && iy >= 1 && iy <= a.ny;
  const bool sea = in_grid && a.mapsta[(ix - 1) * a.ny + (iy - 1)] > 0;
  const float* __restrict__ A = a.va + static_cast<size_t>(jsea) * a.nspec;  // A(ITH,IK)
  auto AA = [&](int ith, int ik) { return A[(ith - 1) + (ik - 1) * nth]; };
  auto cg = [&](int ik) { return a.cg[static_cast<size_t>(isea) * nk2 + ik]; };
  auto wn = [&](int ik) { return a.wn[static_cast<size_t>(isea) * nk2 + ik]; };
  float* const EBD = a.ebd + static_cast<size_t>(j0) * nk;

  // 1. This point's share of the accumulators.
  float et = zero, et02 = zero, ewn = zero, etr = zero, et1 = zero, eet1 = zero;
  float etx = zero, ety = zero, etxx = zero, etyy = zero, etxy = zero;
  float abr = zero, aba = zero, abd = zero, ubr = zero, uba = zero, ubd = zero;
  float sxx = zero, syy = zero, sxy = zero, ussx = zero, ussy = zero, tusx = zero, tusy = zero;
  float mscx = zero, mscy = zero, mscd = zero, prms = zero, tpms = zero, ettpmm = zero;
  float etf = zero, qk2 = zero, bhd = zero;
  float ab = zero, abx = zero, aby = zero, abx2 = zero, aby2 = zero, ab2x = zero, ab2y = zero;
  float abxx = zero, abyy = zero, abxy = zero, abyx = zero, abst = zero, qk1 = zero;

  // 2. The band sums per IK and their integrals.
  for (int ik = 1; ik <= nk; ++ik) {
    ab = zero; abx = zero; aby = zero; abx2 = zero; aby2 = zero; ab2x = zero; ab2y = zero;
    abxx = zero; abyy = zero; abxy = zero; abyx = zero; abst = zero; qk1 = zero;
    const float cgk = cg(ik), wnk = wn(ik), sigk = a.sig[ik];
    for (int ith = 1; ith <= nth; ++ith) {
      const float aj = AA(ith, ik);
      const float ec = a.ecos[ith - 1], es = a.esin[ith - 1], c2 = a.ec2[ith - 1],
                  s2 = a.es2[ith - 1], sc = a.esc[ith - 1];
      ab = ab + aj;
      abx = abx + aj * ec;
      aby = aby + aj * es;
      abx2 = abx2 + aj * c2;
      aby2 = aby2 + aj * s2;
      ab2x = ab2x + aj * (two * c2 - one);
      ab2y = ab2y + aj * (two * sc);
      abyx = abyx + aj * sc;
      if (ith <= nth / 2) {
        const float ah = AA(ith + nth / 2, ik);
        abst = abst + aj * ah;
        const float q = aj + ah;
        qk1 = qk1 + q * q;
      }
      const float factor = gt_sel(cgk / sigk * wnk, half);
      abxx = abxx + ((one + c2) * factor - half) * aj;
      abyy = abyy + ((one + s2) * factor - half) * aj;
      abxy = abxy + sc * factor * aj;
    }
    const float dsik = a.dsii[ik - 1];
    const float factor = a.dden[ik - 1] / cgk;
    float ebd = ab * factor;
    et = et + ebd;
    etf = etf + ebd * cgk;
    ewn = ewn + ebd / wnk;
    etr = etr + ebd / sigk;
    et1 = et1 + ebd * sigk;
    eet1 = eet1 + ebd * ebd * sigk / dsik;
    et02 = et02 + ebd * (sigk * sigk);
    etx = etx + abx * factor;
    ety = ety + aby * factor;
    tusx = tusx + abx * factor * kGrav * wnk / sigk;
    tusy = tusy + aby * factor * kGrav * wnk / sigk;
    const float wn2 = wnk * wnk;
    etxx = etxx + abx2 * factor * wn2;
    qk2 = qk2 + qk1 * factor * sigk / wnk;
    etyy = etyy + aby2 * factor * wn2;
    etxy = etxy + abyx * factor * wn2;

    const float jac = kTpi * sigk / cgk;
    const float factor2 = two * a.dth / kTpi2 * sigk * (jac * jac) * abst;
    prms = prms + factor2 * two * dsik;
    if (a.f69 && ik >= a.p2msf2 && ik <= a.p2msf3)
      put(a.f[OG_P2SMS], j0 + static_cast<size_t>(ik - a.p2msf2) * a.nfld, factor2 * two * kTpi);
    if (factor2 > ettpmm) {
      ettpmm = factor2;
      tpms = kTpi / sigk;
    }
    if (ik == nk) {
      const float s2 = sigk * sigk;
      const float s5 = s2 * sigk * s2;
      const float fac5 = s5 / kGrav2 / dsik;
      const float ma = abx2 * factor * fac5;
      const float mc = aby2 * factor * fac5;
      const float mb = abyx * factor * fac5;
      mscd = half * dm::atan2f(two * mb, ma - mc);
      float cs, sn;
      dm::sincosf(mscd, &sn, &cs);
      mscx = ma * (cs * cs) + two * mb * sn * cs + ma * (sn * sn);
      mscy = mc * (cs * cs) - two * mb * sn * cs + ma * (sn * sn);
    }

    const float kd = gt_sel(wnk * a.dw[isea], 0.001f);
    float ussco;
    if (kd < 6.0f) {
      const float sh = dm::sinhf(kd);
      const float fkd = factor / (sh * sh);
      abr = abr + ab * fkd;
      aba = aba + abx * fkd;
      abd = abd + aby * fkd;
      const float sg2 = sigk * sigk;
      ubr = ubr + ab * sg2 * fkd;
      uba = uba + abx * sg2 * fkd;
      ubd = ubd + aby * sg2 * fkd;
      ussco = fkd * sigk * wnk * dm::coshf(two * kd);
      bhd = bhd + kGrav * wnk * ebd / dm::sinhf(two * kd);
    } else {
      ussco = factor * sigk * two * wnk;
    }
    abxx = gt_sel(abxx, zero) * factor;
    abyy = gt_sel(zero, abyy) * factor;
    abxy = abxy * factor;
    sxx = sxx + abxx;
    syy = syy + abyy;
    sxy = sxy + abxy;
    ebd = ebd / dsik;
    EBD[ik - 1] = ebd;
    if (a.f3[0] && ik >= a.e3df2[0] && ik <= a.e3df3[0])
      put(a.f[OG_EF], j0 + static_cast<size_t>(ik - a.e3df2[0]) * a.nfld, ebd * kTpi);
    ussx = ussx + abx * ussco;
    ussy = ussy + aby * ussco;
    if (a.f3[1] && ik >= a.e3df2[1] && ik <= a.e3df3[1])
      put(a.f[OG_TH1M], j0 + static_cast<size_t>(ik - a.e3df2[1]) * a.nfld,
          fmodf(630.0f - kRade * dm::atan2f(aby, abx), 360.0f));
    const float tiny = 1E-20f;
    const float abm = (a.ompg || a.f3[4]) ? gt_sel(ab, tiny) : gt_sel(tiny, ab);
    const float m1 = sqrtf(abx * abx + aby * aby) / abm;
    if (a.f3[2] && ik >= a.e3df2[2] && ik <= a.e3df3[2])
      put(a.f[OG_STH1M], j0 + static_cast<size_t>(ik - a.e3df2[2]) * a.nfld,
          sqrtf(fabsf(two * (one - m1))) * kRade);
    if (a.f3[3] && ik >= a.e3df2[3] && ik <= a.e3df3[3])
      put(a.f[OG_TH2M], j0 + static_cast<size_t>(ik - a.e3df2[3]) * a.nfld,
          fmodf(270.0f - kRadeHalf * dm::atan2f(ab2y, ab2x), 180.0f));
    const float m2 = sqrtf(ab2x * ab2x + ab2y * ab2y) / abm;
    if (a.f3[4] && ik >= a.e3df2[4] && ik <= a.e3df3[4])
      put(a.f[OG_STH2M], j0 + static_cast<size_t>(ik - a.e3df2[4]) * a.nfld,
          sqrtf(fabsf(half * (one - m2))) * kRade);
  }

  // Space-time extremes, on ET, ET02, ET1, ETX, ETY before the tail of 3.b.
  if (a.ste) {
    const float undef = a.undef;
    float thmp = undef;
    if (sea && fabsf(etx) + fabsf(ety) > k1em7) thmp = dm::atan2f(ety, etx);
    float sth, cth;
    dm::sincosf(thmp, &sth, &cth);

    float mssxm = zero, mssym = zero, mssxtm = zero, mssytm = zero, mssxym = zero;
    for (int ik = 1; ik <= nk; ++ik) {
      float abx2m = zero, aby2m = zero, abxm = zero, abym = zero, abxym = zero;
      for (int ith = 1; ith <= nth; ++ith) {
        const float aj = AA(ith, ik);
        const float ec = a.ecos[ith - 1], es = a.esin[ith - 1];
        const float u = ec * cth + es * sth;
        const float v = es * cth - ec * sth;
        abx2m = abx2m + aj * (u * u);
        aby2m = aby2m + aj * (v * v);
        abxm = abxm + aj * u;
        abym = abym + aj * v;
        abxym = abxym + aj * u * v;
      }
      const float wnk = wn(ik);
      const float factor = a.dden[ik - 1] / cg(ik);
      const float wn2 = wnk * wnk;
      mssxm = mssxm + abx2m * factor * wn2;
      mssym = mssym + aby2m * factor * wn2;
      mssxtm = mssxtm + abxm * factor * wnk * a.sig[ik];
      mssytm = mssytm + abym * factor * wnk * a.sig[ik];
      mssxym = mssxym + abxym * factor * wn2;
    }

    float t02p = undef, wl02x = undef, wl02y = undef, alpxt = undef, alpyt = undef,
          alpxy = undef;
    float nv = undef, ns = undef, nb = undef, mu = undef, ni = undef, mode = undef;
    if (et02 > k1em7) t02p = kTpi * sqrtf(et / et02);
    if (mssxm > k1em7) wl02x = kTpi * sqrtf(et / mssxm);
    if (mssym > k1em7) wl02y = kTpi * sqrtf(et / mssym);
    if (mssxm > k1em7 && et02 > k1em7) alpxt = mssxtm / sqrtf(mssxm * et02);
    if (mssym > k1em7 && et02 > k1em7) alpyt = mssytm / sqrtf(mssym * et02);
    if (mssxm > k1em7 && mssym > k1em7) alpxy = mssxym / sqrtf(mssxm * mssym);

    float stex = zero, stey = zero;
    if (a.stexu > zero && a.steyu > zero) {
      stex = a.stexu;
      stey = a.steyu;
    }
    const float sted = gt_sel(a.stedu, zero);

    if (wl02x > k1em7 && wl02y > k1em7 && t02p > k1em7) {
      const float ax2 = alpxt * alpxt, ay2 = alpyt * alpyt, axy2 = alpxy * alpxy;
      nv = kTpi * (stex * stey * sted) / (wl02x * wl02y * t02p) *
           sqrtf(one - ax2 - ay2 - axy2 + two * alpxt * alpyt * alpxy);
      ns = kSqrtTpi * ((stex * sted) / (wl02x * t02p) * sqrtf(one - ax2) +
                       (stey * sted) / (wl02y * t02p) * sqrtf(one - ay2) +
                       (stex * stey) / (wl02x * wl02y) * sqrtf(one - axy2));
      nb = stex / wl02x + stey / wl02y + sted / t02p;
    }
    if (et1 > k1em7) ni = sqrtf(et * et02 / (et1 * et1) - one);
    if (et > k1em7) mu = et1 * et1 / kGrav * dm::powf(et, -1.5f) * (one - ni + ni * ni);

    if (stex == zero && stey == zero) {
      mode = sqrtf(two * dm::logf(nb));
    } else if (sted == zero) {
      const float t = two * dm::logf(ns);
      mode = sqrtf(t + dm::logf(t + dm::logf(t)));
    } else if (wl02x > k1em7 && wl02y > k1em7 && t02p > k1em7) {
      const float t = two * dm::logf(nv);
      mode = sqrtf(t + two * dm::logf(t + two * dm::logf(t)));
    }

    const float sqet = sqrtf(et);
    const float mode2 = mode * mode;
    const float den = mode - (two * nv * mode + ns) / (nv * mode2 + ns * mode + nb);
    const float mum = one + mu * mode;
    put(a.f[OG_STMAXE], j0, sqet * (mode + half * mu * mode2 + 0.5772f * mum / den));
    put(a.f[OG_STMAXD], j0, sqet * (kPi * mum / kSqrt6 / den));

    float phist = zero;
    if (t02p > k1em7) {
      float phi[21];
#pragma unroll
      for (int itl = 0; itl < 21; ++itl) phi[itl] = zero;
      float tlphi = 0.3f * t02p;
      const float xfr = a.xfr, x2 = xfr * xfr, x3 = xfr * x2;
#pragma unroll
      for (int itl = 0; itl < 21; ++itl) {
        for (int ik = 1; ik <= nk - 3; ik += 4) {
          const float sigk = a.sig[ik];
          phi[itl] = phi[itl] + (x3 * EBD[ik + 2] * cosf_(x3 * sigk * tlphi) +
                                 x2 * EBD[ik + 1] * cosf_(x2 * sigk * tlphi) +
                                 xfr * EBD[ik] * cosf_(xfr * sigk * tlphi) +
                                 EBD[ik - 1] * cosf_(sigk * tlphi)) *
                                    a.dsii[ik - 1];
        }
        tlphi = tlphi + t02p / 20.0f;
      }
#pragma unroll
      for (int itl = 0; itl < 21; ++itl) phi[itl] = phi[itl] / et;
      // MINVAL: from the first element that is not a NaN, then a < min ? a : min; 21 NaNs
      // give NaN.
      float mn = __int_as_float(0x7fc00000);
      bool found = false;
#pragma unroll
      for (int m = 0; m < 21; ++m) {
        if (found) {
          mn = lt_sel(phi[m], mn);
        } else if (phi[m] == phi[m]) {
          mn = phi[m];
          found = true;
        }
      }
      phist = fabsf(mn);
    }

    const float stmaxel = sqet * (mode + 0.5772f / den);
    const float stmaxdl = sqet * (kPiSqrt6 / den);
    put(a.f[OG_HCMAXE], j0, stmaxel * (one + phist));
    put(a.f[OG_HCMAXD], j0, stmaxdl * (one + phist));
    const float sq2 = sqrtf(two * (one + phist));
    put(a.f[OG_HMAXE], j0, stmaxel * sq2);
    put(a.f[OG_HMAXD], j0, stmaxdl * sq2);
  }

  // 3.a
  {
    const float mssd = half * dm::atan2f(two * etxy, etxx - etyy);
    float cs, sn;
    dm::sincosf(mssd, &sn, &cs);
    put(a.f[OG_MSSX], j0, etxx * (cs * cs) + two * etxy * sn * cs + etyy * (sn * sn));
    put(a.f[OG_MSSY], j0, etyy * (cs * cs) - two * etxy * sn * cs + etxx * (sn * sn));
    put(a.f[OG_MSSD], j0, mssd);
  }

  // 3.b, the tail beyond SIG(NK): AB, ABX, ABY, ABXX, ABYY, ABXY are those of IK = NK.
  const float signk = a.sig[nk];
  const float cgnk = cg(nk);
  const float ft1 = 0.3333f * (signk * signk) * a.dth * signk;
  const float eband = ab / cgnk;
  et = et + a.fte * eband;
  ewn = ewn + a.ftwl * eband;
  etf = etf + kGrav * a.fttr * eband;
  etr = etr + a.fttr * eband;
  et1 = et1 + ft1 * eband;
  const float sn2 = signk * signk;
  et02 = et02 + eband * half * (sn2 * sn2) * a.dth;
  etx = etx + a.fte * abx / cgnk;
  ety = ety + a.fte * aby / cgnk;
  sxx = sxx + a.fte * abxx / cgnk;
  syy = syy + a.fte * abyy / cgnk;
  sxy = sxy + a.fte * abxy / cgnk;

  put(a.f[OG_SXX], j0, sxx * kDwat * kGrav);
  put(a.f[OG_SYY], j0, syy * kDwat * kGrav);
  put(a.f[OG_SXY], j0, sxy * kDwat * kGrav);

  if (sea) {
    put(a.f[OG_HS], j0, 4.0f * sqrtf(et));
    if (et > k1em7) {
      const float et2 = et * et;
      put(a.f[OG_QP], j0, (two / et2) * eet1);
      put(a.f[OG_WLM], j0, ewn / et * kTpi);
      put(a.f[OG_T0M1], j0, etr / et * kTpi);
      float ths = kRade * sqrtf(gt_sel(two * (one - sqrtf(gt_sel((etx * etx + ety * ety) / et2,
                                                                  zero))),
                                        zero));
      if (ths < kRade001 * a.dth) ths = zero;
      put(a.f[OG_THS], j0, ths);
      put(a.f[OG_QKK], j0, sqrtf(half * qk2) / et);
    } else {
      put(a.f[OG_WLM], j0, zero);
      put(a.f[OG_T0M1], j0, kTpi / signk);
      put(a.f[OG_THS], j0, zero);
    }
    put(a.f[OG_THM], j0, (fabsf(etx) + fabsf(ety) > k1em7) ? dm::atan2f(ety, etx) : zero);
    abr = sqrtf(two * gt_sel(zero, abr));
    abd = (abr >= k1em7) ? dm::atan2f(abd, aba) : zero;
    aba = abr;
    ubr = sqrtf(two * gt_sel(zero, ubr));
    ubd = (ubr >= k1em7) ? dm::atan2f(ubd, uba) : zero;
    uba = ubr;
    put(a.f[OG_CGE], j0, kDwatGrav * etf);
    if (et02 > k1em7 && et > zero) {
      put(a.f[OG_T02], j0, kTpi * sqrtf(et / et02));
      put(a.f[OG_T01], j0, kTpi * et / et1);
    } else {
      const float t02 = kTpi / signk;
      put(a.f[OG_T02], j0, t02);
      put(a.f[OG_T01], j0, t02);
    }
  }
  put(a.f[OG_ABA], j0, aba);
  put(a.f[OG_ABD], j0, abd);
  put(a.f[OG_UBA], j0, uba);
  put(a.f[OG_UBD], j0, ubd);
  put(a.f[OG_USSX], j0, ussx);
  put(a.f[OG_USSY], j0, ussy);
  put(a.f[OG_TUSX], j0, tusx);
  put(a.f[OG_TUSY], j0, tusy);
  put(a.f[OG_MSCX], j0, mscx);
  put(a.f[OG_MSCY], j0, mscy);
  put(a.f[OG_MSCD], j0, mscd);
  put(a.f[OG_PRMS], j0, prms);
  put(a.f[OG_TPMS], j0, tpms);
  put(a.f[OG_BHD], j0, bhd);

  // 4. The peak frequency FP0 and its direction THP0.
  float ec = EBD[nk - 1];
  int ikp0 = nk;
  float fp0 = a.undef, thp0 = a.undef;
  for (int ik = nk - 1; ik >= 1; --ik) {
    if (ec < EBD[ik - 1]) {
      ec = EBD[ik - 1];
      ikp0 = ik;
    }
  }
  if (ikp0 != nk) fp0 = a.sig[ikp0] * kTpiInv;
  const float xl = one / a.xfr - one, xh = a.xfr - one;
  const float xl2 = xl * xl, xh2 = xh * xh;
  if (ikp0 != nk) {
    const float e0 = EBD[ikp0 - 1];
    const float el = (ikp0 == 1) ? -e0 : EBD[ikp0 - 2] - e0;
    const float eh = EBD[ikp0] - e0;
    const float denom = xl * eh - xh * el;
    fp0 = fp0 * (one + half * (xl2 * eh - xh2 * el) /
                           copysignf(gt_sel(fabsf(denom), 1.E-15f), denom));
  }
  float etxp = zero, etyp = zero;
  if (ikp0 != nk) {
    for (int ith = 1; ith <= nth; ++ith) {
      etxp = etxp + AA(ith, ikp0) * a.ecos[ith - 1];
      etyp = etyp + AA(ith, ikp0) * a.esin[ith - 1];
    }
  }
  if (fabsf(etxp) + fabsf(etyp) > k1em7 && fp0 != a.undef) thp0 = dm::atan2f(etyp, etxp);
  if (!sea) {
    fp0 = a.undef;
    thp0 = a.undef;
  }
  put(a.f[OG_FP0], j0, fp0);
  put(a.f[OG_THP0], j0, thp0);
}

#undef F1

/// 6.a: UNDEF in every partition field over its NROW rows.
__global__ void outg_part_init_kernel(OutgPartArgs a) {
  const int ncol = a.noswll + 1;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.nrow; j += gridDim.x * blockDim.x) {
    for (int c = 0; c < ncol; ++c)
      for (int k = 0; k < 15; ++k) a.f[k][j + static_cast<size_t>(c) * a.nrow] = a.undef;
    a.f[15][j] = a.undef;
    a.f[16][j] = a.undef;
  }
}

/// 6.b: PNR and PWST of each sea point and its partitions' rows of DTPRT, the wind sea first
/// when its wind-sea fraction (DTPRT(6,.)) reaches WSCUT.
__global__ void outg_part_kernel(OutgPartArgs a) {
  const int jsea = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (jsea > a.nseal) return;
  const int j0 = jsea - 1, isea = jsea;
  const int ix = a.mapsf[isea - 1], iy = a.mapsf[a.nsea + isea - 1];
  const bool sea = a.mapsta[(ix - 1) * a.ny + (iy - 1)] > 0;
  const int n1 = a.icprt[j0], n2 = a.icprt[a.nicp + j0];  // ICPRT(JSEA,1:2)
  const size_t nr = a.nrow;
  auto d = [&](int k, int ip) { return a.dtprt[(k - 1) + static_cast<size_t>(ip - 1) * a.dimp]; };
  if (sea) {
    a.f[16][j0] = gt_sel(static_cast<float>(n1 - 1), 0.0f);
    if (n1 >= 1) a.f[15][j0] = d(6, n2);
  }
  if (!(sea && n1 > 1)) return;
  auto copy = [&](int j, int ip) {
    const size_t o = j0 + j * nr;
    a.f[0][o] = d(1, ip);
    a.f[1][o] = d(2, ip);
    a.f[2][o] = d(3, ip);
    if (d(4, ip) != a.undef) a.f[3][o] = (270.0f - d(4, ip)) * kDera;
    a.f[4][o] = d(5, ip);
    a.f[5][o] = d(6, ip);
    if (d(7, ip) != a.undef) a.f[6][o] = (270.0f - d(7, ip)) * kDera;
    a.f[10][o] = d(8, ip);  // PSW
    a.f[8][o] = d(9, ip);   // PPE
    a.f[7][o] = d(10, ip);  // PQP
    a.f[9][o] = d(11, ip);  // PGW
    a.f[11][o] = d(12, ip);
    a.f[12][o] = d(13, ip);
    a.f[13][o] = d(14, ip);
    a.f[14][o] = d(15, ip);
  };
  int i = n2 + 1;
  if (d(6, i) >= a.wscut) {
    copy(0, i);
    i = i + 1;
  }
  for (int j = 1; j <= a.noswll; ++j) {
    if (i > n2 + n1 - 1) break;
    copy(j, i);
    i = i + 1;
  }
}

int blocks_for(long long n, int per) {
  const long long b = (n + per - 1) / per;
  return static_cast<int>(b < 1 ? 1 : (b > 65535 ? 65535 : b));
}

}  // namespace

void launch_outg(const OutgArgs& a, cudaStream_t s) {
  if (a.nfld > 0) outg_init_kernel<<<blocks_for(a.nfld, 256), 256, 0, s>>>(a);
  WWB_CHECK(cudaGetLastError());
  if (a.nseal <= 0) return;
  outg_point_kernel<<<(a.nseal + 127) / 128, 128, 0, s>>>(a);
  WWB_CHECK(cudaGetLastError());
}

void launch_outg_part(const OutgPartArgs& a, cudaStream_t s) {
  if (a.nrow > 0) outg_part_init_kernel<<<blocks_for(a.nrow, 256), 256, 0, s>>>(a);
  WWB_CHECK(cudaGetLastError());
  if (a.nseal <= 0) return;
  outg_part_kernel<<<(a.nseal + 127) / 128, 128, 0, s>>>(a);
  WWB_CHECK(cudaGetLastError());
}

}  // namespace wwb
