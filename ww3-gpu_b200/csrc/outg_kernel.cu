// ww3-gpu_b200/csrc/outg_kernel.cu
// W3OUTG on sm_100a (see outg_kernel.cuh): a CTA takes eight sea points; their per-IK work runs
// one thread per (point, IK) and one thread per point adds it up in the reference's order.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/iogo_w3outg.hpp:198-598 (w3outg_point: sections 2-4 and
// the space-time extremes of w3iogomd.F90:1201-2380), :603-690 (w3outg_part_point, section 6),
// :693-713 (the whole-array assignments of section 1). The sums over ITH (per IK) and over IK
// (per point) are sequential in the reference and stay so: no reduction is reordered. MAX/MIN keep
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

// ---------------------------------------------------------------------------------------------
// W3OUTG with the point's independent work spread over the CTA: P points per CTA; the per-IK
// work of section 2 (the band sums over ITH and every per-IK term) and of the space-time
// extremes (the rotated band sums, the 21 PHI sums) runs one thread per (point, IK) or (point,
// ITL); one thread per point then adds the terms over IK in the reference's order. Every sum keeps
// its order and every term its association, so the bits are those of the one-thread form.
constexpr int kOutgThreads = 128;
constexpr int kRec = 32;  // floats of one (point, IK) record

// Record slots (section 2's per-IK terms; the raw band sums of IK = NK for 3.b and MSC).
enum : int {
  R_EBD = 0, R_ETF, R_EWN, R_ETR, R_ET1, R_EET1, R_ET02, R_ETX, R_ETY, R_TUSX, R_TUSY, R_ETXX,
  R_QK2, R_ETYY, R_ETXY, R_PRMS, R_F2, R_TPMS, R_ABR, R_ABA, R_ABD, R_UBR, R_UBA, R_UBD, R_USSX,
  R_USSY, R_BHD, R_SXX, R_SYY, R_SXY, R_KD6, R_AB
};
static_assert(R_AB < kRec, "record layout");

__global__ void __launch_bounds__(kOutgThreads) outg_cta_kernel(OutgArgs a, int P) {
  extern __shared__ float sm[];
  const float zero = 0.0f, half = 0.5f, one = 1.0f, two = 2.0f, k1em7 = 1.E-7f;
  const int nk = a.nk, nth = a.nth, nk2 = nk + 2, tid = threadIdx.x;
  const int first = blockIdx.x * P;  // the CTA's first point, 0-based
  const int np = min(P, a.nseal - first);
  float* const rec = sm;                                   // [P][nk][kRec]
  float* const rot = rec + static_cast<size_t>(P) * nk * kRec;  // cth, sth, t02p, phi[21]
  auto R = [&](int p, int ik) { return rec + (static_cast<size_t>(p) * nk + (ik - 1)) * kRec; };
  // Per point: cth, sth, t02p, the raw band sums of IK = NK (6), PHI(21).
  auto RT = [&](int p) { return rot + static_cast<size_t>(p) * 32; };

  // Phase A: one thread per (point, IK).
  for (int pair = tid; pair < np * nk; pair += blockDim.x) {
    const int p = pair / nk, ik = pair - p * nk + 1;
    const int j0 = first + p, isea = j0 + 1;
    const float* __restrict__ A = a.va + static_cast<size_t>(isea) * a.nspec + (ik - 1) * nth;
    const float cgk = a.cg[static_cast<size_t>(isea) * nk2 + ik];
    const float wnk = a.wn[static_cast<size_t>(isea) * nk2 + ik];
    const float sigk = a.sig[ik];
    float ab = zero, abx = zero, aby = zero, abx2 = zero, aby2 = zero, ab2x = zero, ab2y = zero;
    float abxx = zero, abyy = zero, abxy = zero, abyx = zero, abst = zero, qk1 = zero;
    for (int ith = 1; ith <= nth; ++ith) {
      const float aj = A[ith - 1];
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
        const float ah = A[ith + nth / 2 - 1];
        abst = abst + aj * ah;
        const float q = aj + ah;
        qk1 = qk1 + q * q;
      }
      const float factor = gt_sel(cgk / sigk * wnk, half);
      abxx = abxx + ((one + c2) * factor - half) * aj;
      abyy = abyy + ((one + s2) * factor - half) * aj;
      abxy = abxy + sc * factor * aj;
    }
    float* const r = R(p, ik);
    const float dsik = a.dsii[ik - 1];
    const float factor = a.dden[ik - 1] / cgk;
    float ebd = ab * factor;
    r[R_EBD] = ebd;
    r[R_ETF] = ebd * cgk;
    r[R_EWN] = ebd / wnk;
    r[R_ETR] = ebd / sigk;
    r[R_ET1] = ebd * sigk;
    r[R_EET1] = ebd * ebd * sigk / dsik;
    r[R_ET02] = ebd * (sigk * sigk);
    r[R_ETX] = abx * factor;
    r[R_ETY] = aby * factor;
    r[R_TUSX] = abx * factor * kGrav * wnk / sigk;
    r[R_TUSY] = aby * factor * kGrav * wnk / sigk;
    const float wn2 = wnk * wnk;
    r[R_ETXX] = abx2 * factor * wn2;
    r[R_QK2] = qk1 * factor * sigk / wnk;
    r[R_ETYY] = aby2 * factor * wn2;
    r[R_ETXY] = abyx * factor * wn2;
    const float jac = kTpi * sigk / cgk;
    const float factor2 = two * a.dth / kTpi2 * sigk * (jac * jac) * abst;
    r[R_PRMS] = factor2 * two * dsik;
    r[R_F2] = factor2;
    r[R_TPMS] = kTpi / sigk;
    if (a.f69 && ik >= a.p2msf2 && ik <= a.p2msf3)
      put(a.f[OG_P2SMS], j0 + static_cast<size_t>(ik - a.p2msf2) * a.nfld, factor2 * two * kTpi);
    const float kd = gt_sel(wnk * a.dw[isea], 0.001f);
    float ussco;
    r[R_KD6] = kd < 6.0f ? one : zero;
    if (kd < 6.0f) {
      const float sh = dm::sinhf(kd);
      const float fkd = factor / (sh * sh);
      r[R_ABR] = ab * fkd;
      r[R_ABA] = abx * fkd;
      r[R_ABD] = aby * fkd;
      const float sg2 = sigk * sigk;
      r[R_UBR] = ab * sg2 * fkd;
      r[R_UBA] = abx * sg2 * fkd;
      r[R_UBD] = aby * sg2 * fkd;
      ussco = fkd * sigk * wnk * dm::coshf(two * kd);
      r[R_BHD] = kGrav * wnk * ebd / dm::sinhf(two * kd);
    } else {
      ussco = factor * sigk * two * wnk;
    }
    abxx = gt_sel(abxx, zero) * factor;
    abyy = gt_sel(zero, abyy) * factor;
    abxy = abxy * factor;
    r[R_SXX] = abxx;
    r[R_SYY] = abyy;
    r[R_SXY] = abxy;
    ebd = ebd / dsik;
    a.ebd[static_cast<size_t>(j0) * nk + (ik - 1)] = ebd;
    if (a.f3[0] && ik >= a.e3df2[0] && ik <= a.e3df3[0])
      put(a.f[OG_EF], j0 + static_cast<size_t>(ik - a.e3df2[0]) * a.nfld, ebd * kTpi);
    r[R_USSX] = abx * ussco;
    r[R_USSY] = aby * ussco;
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
    if (ik == nk) {  // the raw band sums of IK = NK (3.b's tail and MSC)
      float* const t = RT(p);
      t[3] = ab;
      t[4] = abx;
      t[5] = aby;
      t[6] = abx2;
      t[7] = aby2;
      t[8] = abyx;
    }
  }
  __syncthreads();

  // Phase B: one thread per point adds the terms over IK in order.
  const bool mine = tid < np;
  const int p = tid, j0 = first + tid, isea = j0 + 1;
  float et = zero, et02 = zero, ewn = zero, etr = zero, et1 = zero, eet1 = zero;
  float etx = zero, ety = zero, etxx = zero, etyy = zero, etxy = zero;
  float abr = zero, aba = zero, abd = zero, ubr = zero, uba = zero, ubd = zero;
  float sxx = zero, syy = zero, sxy = zero, ussx = zero, ussy = zero, tusx = zero, tusy = zero;
  float mscx = zero, mscy = zero, mscd = zero, prms = zero, tpms = zero, ettpmm = zero;
  float etf = zero, qk2 = zero, bhd = zero;
  bool sea = false;
  if (mine) {
    const int ix = a.mapsf[isea - 1], iy = a.mapsf[a.nsea + isea - 1];
    const bool in_grid = ix >= 1 && ix <= a.nx && iy >= 1 && iy <= a.ny;
    sea = in_grid && a.mapsta[(ix - 1) * a.ny + (iy - 1)] > 0;
    for (int ik = 1; ik <= nk; ++ik) {
      const float* const r = R(p, ik);
      et = et + r[R_EBD];
      etf = etf + r[R_ETF];
      ewn = ewn + r[R_EWN];
      etr = etr + r[R_ETR];
      et1 = et1 + r[R_ET1];
      eet1 = eet1 + r[R_EET1];
      et02 = et02 + r[R_ET02];
      etx = etx + r[R_ETX];
      ety = ety + r[R_ETY];
      tusx = tusx + r[R_TUSX];
      tusy = tusy + r[R_TUSY];
      etxx = etxx + r[R_ETXX];
      qk2 = qk2 + r[R_QK2];
      etyy = etyy + r[R_ETYY];
      etxy = etxy + r[R_ETXY];
      prms = prms + r[R_PRMS];
      if (r[R_F2] > ettpmm) {
        ettpmm = r[R_F2];
        tpms = r[R_TPMS];
      }
      if (r[R_KD6] != zero) {
        abr = abr + r[R_ABR];
        aba = aba + r[R_ABA];
        abd = abd + r[R_ABD];
        ubr = ubr + r[R_UBR];
        uba = uba + r[R_UBA];
        ubd = ubd + r[R_UBD];
        bhd = bhd + r[R_BHD];
      }
      sxx = sxx + r[R_SXX];
      syy = syy + r[R_SYY];
      sxy = sxy + r[R_SXY];
      ussx = ussx + r[R_USSX];
      ussy = ussy + r[R_USSY];
    }
    {  // MSC from the band sums of IK = NK
      const float* const t = RT(p);
      const float sigk = a.sig[nk], dsik = a.dsii[nk - 1];
      const float factor = a.dden[nk - 1] / a.cg[static_cast<size_t>(isea) * nk2 + nk];
      const float s2 = sigk * sigk;
      const float s5 = s2 * sigk * s2;
      const float fac5 = s5 / kGrav2 / dsik;
      const float ma = t[6] * factor * fac5;
      const float mc = t[7] * factor * fac5;
      const float mb = t[8] * factor * fac5;
      mscd = half * dm::atan2f(two * mb, ma - mc);
      float cs, sn;
      dm::sincosf(mscd, &sn, &cs);
      mscx = ma * (cs * cs) + two * mb * sn * cs + ma * (sn * sn);
      mscy = mc * (cs * cs) - two * mb * sn * cs + ma * (sn * sn);
    }
    if (a.ste) {
      float thmp = a.undef;
      if (sea && fabsf(etx) + fabsf(ety) > k1em7) thmp = dm::atan2f(ety, etx);
      float sth, cth;
      dm::sincosf(thmp, &sth, &cth);
      RT(p)[0] = cth;
      RT(p)[1] = sth;
    }
  }
  __syncthreads();

  // Phase C: the rotated band sums, one thread per (point, IK), into the records.
  if (a.ste) {
    for (int pair = tid; pair < np * nk; pair += blockDim.x) {
      const int q = pair / nk, ik = pair - q * nk + 1;
      const int jq = first + q, iq = jq + 1;
      const float* __restrict__ A = a.va + static_cast<size_t>(iq) * a.nspec + (ik - 1) * nth;
      const float cth = RT(q)[0], sth = RT(q)[1];
      float abx2m = zero, aby2m = zero, abxm = zero, abym = zero, abxym = zero;
      for (int ith = 1; ith <= nth; ++ith) {
        const float aj = A[ith - 1];
        const float ec = a.ecos[ith - 1], es = a.esin[ith - 1];
        const float u = ec * cth + es * sth;
        const float v = es * cth - ec * sth;
        abx2m = abx2m + aj * (u * u);
        aby2m = aby2m + aj * (v * v);
        abxm = abxm + aj * u;
        abym = abym + aj * v;
        abxym = abxym + aj * u * v;
      }
      const float wnk = a.wn[static_cast<size_t>(iq) * nk2 + ik];
      const float factor = a.dden[ik - 1] / a.cg[static_cast<size_t>(iq) * nk2 + ik];
      const float wn2 = wnk * wnk;
      float* const r = R(q, ik);
      r[0] = abx2m * factor * wn2;
      r[1] = aby2m * factor * wn2;
      r[2] = abxm * factor * wnk * a.sig[ik];
      r[3] = abym * factor * wnk * a.sig[ik];
      r[4] = abxym * factor * wn2;
    }
  }
  __syncthreads();

  // Phase D: the space-time extremes' scalars of each point.
  float sqet = zero, mode = zero, den = zero;
  if (a.ste && mine) {
    const float undef = a.undef;
    float mssxm = zero, mssym = zero, mssxtm = zero, mssytm = zero, mssxym = zero;
    for (int ik = 1; ik <= nk; ++ik) {
      const float* const r = R(p, ik);
      mssxm = mssxm + r[0];
      mssym = mssym + r[1];
      mssxtm = mssxtm + r[2];
      mssytm = mssytm + r[3];
      mssxym = mssxym + r[4];
    }
    float t02p = undef, wl02x = undef, wl02y = undef, alpxt = undef, alpyt = undef,
          alpxy = undef;
    float nv = undef, ns = undef, nb = undef, mu = undef, ni = undef;
    mode = undef;
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
    sqet = sqrtf(et);
    const float mode2 = mode * mode;
    den = mode - (two * nv * mode + ns) / (nv * mode2 + ns * mode + nb);
    const float mum = one + mu * mode;
    put(a.f[OG_STMAXE], j0, sqet * (mode + half * mu * mode2 + 0.5772f * mum / den));
    put(a.f[OG_STMAXD], j0, sqet * (kPi * mum / kSqrt6 / den));
    RT(p)[2] = t02p;
  }
  __syncthreads();

  // Phase E: PHI(ITL), one thread per (point, ITL); TLPHI is stepped as the reference steps it.
  if (a.ste) {
    for (int pair = tid; pair < np * 21; pair += blockDim.x) {
      const int q = pair / 21, itl = pair - q * 21;
      const float t02p = RT(q)[2];
      if (!(t02p > k1em7)) continue;
      const float* const ebd = a.ebd + static_cast<size_t>(first + q) * nk;
      float tlphi = 0.3f * t02p;
      for (int k = 0; k < itl; ++k) tlphi = tlphi + t02p / 20.0f;
      const float xfr = a.xfr, x2 = xfr * xfr, x3 = xfr * x2;
      float ph = zero;
      for (int ik = 1; ik <= nk - 3; ik += 4) {
        const float sigk = a.sig[ik];
        ph = ph + (x3 * ebd[ik + 2] * cosf_(x3 * sigk * tlphi) +
                   x2 * ebd[ik + 1] * cosf_(x2 * sigk * tlphi) +
                   xfr * ebd[ik] * cosf_(xfr * sigk * tlphi) + ebd[ik - 1] * cosf_(sigk * tlphi)) *
                      a.dsii[ik - 1];
      }
      RT(q)[9 + itl] = ph;
    }
  }
  __syncthreads();
  if (!mine) return;

  // Phase F: the rest of the point (one thread each).
  if (a.ste) {
    float phist = zero;
    const float t02p = RT(p)[2];
    if (t02p > k1em7) {
      // MINVAL: from the first element that is not a NaN, then a < min ? a : min.
      float mn = __int_as_float(0x7fc00000);
      bool found = false;
      for (int m = 0; m < 21; ++m) {
        const float ph = RT(p)[9 + m] / et;
        if (found) {
          mn = lt_sel(ph, mn);
        } else if (ph == ph) {
          mn = ph;
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
  // The band sums of IK = NK that 3.b's tail reads.
  const float ab = RT(p)[3], abx = RT(p)[4], aby = RT(p)[5];
  const float abxx = R(p, nk)[R_SXX], abyy = R(p, nk)[R_SYY], abxy = R(p, nk)[R_SXY];
  const float* __restrict__ A = a.va + static_cast<size_t>(isea) * a.nspec;
  auto AA = [&](int ith, int ik) { return A[(ith - 1) + (ik - 1) * nth]; };
  auto cg = [&](int ik) { return a.cg[static_cast<size_t>(isea) * nk2 + ik]; };
  const float* const EBD = a.ebd + static_cast<size_t>(j0) * nk;

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
  // Eight points per CTA: their (point, IK) records take about 37 KB at 36 frequencies, so
  // five CTAs share an SM.
  constexpr int kPoints = 8;
  const size_t smem = sizeof(float) * kPoints * (static_cast<size_t>(a.nk) * kRec + 32);
  if (smem > 48 * 1024)
    WWB_CHECK(cudaFuncSetAttribute(outg_cta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
  outg_cta_kernel<<<(a.nseal + kPoints - 1) / kPoints, kOutgThreads, smem, s>>>(a, kPoints);
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
