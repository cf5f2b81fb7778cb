// ww3-gpu_b200/csrc/st4_point.cuh
// WAVEWATCH III's ST4 source terms (W3SIN4, W3SDS4, W3SPR4 with CALC_USTAR) for one sea point,
// run by one CTA, written once for the device and the host.
//
// Each routine is a sequence of phases. A phase is either a strided loop over the CTA's threads
// (PFOR: independent elements, e.g. the directions of one frequency) or a serial stretch on one
// thread (ROLE: every sum whose order the reference fixes, every recurrence over frequency).
// Phases are separated by cta.sync(). Compiled for the host with one "thread" the same source
// runs the phases in order, which is how the CPU tests check the kernels' arithmetic against the
// reference's own build without a GPU.
//
// Arithmetic: the reference's statements (ww3-gpu kokkos/src/ww_kokkos/st4_sin4.hpp:69-630,
// st4_sds4.hpp:120-745, st4_spr4.hpp:40-160, st4_calc_ustar.hpp:36-124; WW3 w3src4md.F90 at
// bb08623a), each with its operand order and rounding: x**4 as (x*x)*(x*x), REAL exponents as
// powf, MAX(a,b) as a > b ? a : b unless a site says otherwise. libm calls go to libm_dev.cuh
// (glibc's bits for expf, logf, powf, sincosf, tanhf, log10f). Two differences from the
// reference's CPU build are inherent and documented at the call sites: atan2f is fdlibm's
// (1-ulp differences from this glibc's on ~0.02 % of arguments), and the five libmvec loops
// (w3src4md.F90:316, :317, :2315, :2500, :2509) use scalar powf/expf in every lane.
#pragma once

#include <stdint.h>

#include "libm_dev.cuh"
#include "st4_params.hpp"

#if defined(__CUDACC__)
#define WWB_PD __host__ __device__ __forceinline__
#define WWB_PN __host__ __device__ __noinline__  // the large routines: called, not inlined
#define WWB_PRAGMA(x) _Pragma(#x)
#define WWB_UNROLL(n) WWB_PRAGMA(unroll n)
#else
#define WWB_PD inline
#define WWB_PN inline
#define WWB_UNROLL(n)
#endif

namespace wwb {
namespace pt {

/// The threads of one CTA working on one point (on the host: one thread).
struct Cta {
  int tid, nthr;
  WWB_PD void sync() const {
#if defined(__CUDA_ARCH__)
    __syncthreads();
#endif
  }
  /// Whether this thread runs serial role r: role r is the first thread of warp r (so roles of
  /// one phase run side by side, not serialized within a warp); all on thread 0 of a one-thread
  /// CTA.
  WWB_PD bool role(int r) const { return tid == (32 * r) % nthr; }
};

#define PFOR(i, n) for (int i = cta.tid; i < (n); i += cta.nthr)

// CONSTANTS (constants.F90:62-95) as float expressions, each operation rounded to float.
constexpr float kPi = static_cast<float>(3.141592653589793);
constexpr float kTpi = 2.0f * kPi;
constexpr float kTpiInv = 1.0f / kTpi;
constexpr float kGrav = 9.806f;
constexpr float kDwat = 1000.0f;
constexpr float kNuAir = 1.4E-5f;
constexpr float kKappa = 0.40f;
constexpr float kAbMin = -1.0f;

WWB_PD float max_r(float a, float b) { return a > b ? a : b; }
WWB_PD float min_r(float a, float b) { return a < b ? a : b; }
WWB_PD int max_i(int a, int b) { return a > b ? a : b; }
WWB_PD int min_i(int a, int b) { return a < b ? a : b; }

/// INT(x) as gfortran's cvttss2si: truncation, INT_MIN for NaN or out of range.
WWB_PD int fint(float x) {
  return (x > -2147483904.0f && x < 2147483648.0f) ? static_cast<int>(x)
                                                   : static_cast<int>(0x80000000u);
}
/// NINT(x): round half away from zero, NaN / out of range 0.
WWB_PD int nint(float x) {
  const float r = roundf(x);
  return (r > -9.2233715e18f && r < 9.2233715e18f) ? static_cast<int>(static_cast<long long>(r))
                                                   : 0;
}
WWB_PD float fabs_f(float x) { return fabsf(x); }
/// A load of a large read-only table that is streamed once per use (CUMULW): it is not kept in
/// L1, so the small tables and the stack that the serial chains read stay there.
WWB_PD float ld_stream(const float* p) {
#if defined(__CUDA_ARCH__)
  float v;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
#else
  return *p;
#endif
}
WWB_PD float sqrt_f(float x) { return sqrtf(x); }
WWB_PD bool isnan_f(float x) { return x != x; }

/// The arrays ST4 reads (st4_arrays.hpp:41-81), as pointers with their registered extents.
/// Every pointer is at the Fortran lower bound: sig[ik] is SIG(IK) (SIG(0:MK+1)), dsip[ik] is
/// DSIP(IK), esin[is-1] is ESIN(IS), and so on.
struct Fields {
  const float *sig, *sig2, *dsip, *dden, *dden2, *esin, *ecos, *th;
  const float* satw_t;  ///< SATWEIGHTS transposed: (ith-1) + (j-1)*sat_ld
  const int* sati_t;
  int nsat, sat_ld;
  const float* cumulw;  ///< CUMULW transposed: CUMULW(i,j) = cumulw[(j-1) + (i-1)*cumulw_ld]
  int cumulw_ld;
  const float *dcki, *qbi;  ///< (NKHS, NKD)
  const int* iktab;         ///< IKTAB(ik,id) = iktab[(ik-1) + (id-1)*iktab_ld]
  int iktab_ld;
  const float *taut, *tauhft, *tauhft2, *fwtable;
  WWB_PD float taut_at(int i, int j) const { return taut[i + j * (st4::kItauMax + 1)]; }
  WWB_PD float tauhft_at(int i, int j) const { return tauhft[i + j * (st4::kIustar + 1)]; }
  WWB_PD float tauhft2_at(int i, int j, int k) const {
    return tauhft2[i + (st4::kIustar + 1) * (j + (st4::kIalpha + 1) * k)];
  }
};

// ===================================================================================== W3SIN4
// Constants gfortran folds (st4_sin4.hpp:29-45).
constexpr float kKappa2 = kKappa * kKappa;
constexpr float kZ0viscNum = 0.1f * kNuAir;
constexpr float kTwoNuAir = 2.0f * kNuAir;
constexpr float kGrav2Tpi = (kGrav * kGrav) * kTpi;
constexpr float kLogTpiOver005 = 7.1361942291259765625e+0f;  // LOG(TPI/0.005), folded
constexpr float kEps1 = 0.00001f, kEps2 = 0.000001f;
constexpr float kEps2Sq = kEps2 * kEps2;
constexpr int kJtot = 50;
constexpr float kKm = 363.0f, kCmm = 0.2325f;

/// The point's W3SIN4 state that crosses phases (shared by the CTA).
struct Sin4Sh {
  float const1, const0, uorb, pturb, pvisc, fw, fu, fud, ustarsigma;
  float ust, taux, tauy, cosu, sinu, ustp, usdirp;
  float ss[3][2], sn[3][2];
  float term[2][3][128];  ///< double-buffered per-direction stress terms (c, s, sign), NTH <= 128
  float tail[7][kJtot];   ///< the analytic tail's terms that do not depend on USTR, per J
};

/// Reals of W3SIN4's NK work: EB and the six per-IK factors of the stress scan.
WWB_PD int sin4_nk_work(const st4::Params& p) { return 7 * p.nk; }


/// Reals of the DSTAB work W3SIN4 needs (3 x NSPEC).
WWB_PD int sin4_work(const st4::Params& p) { return 3 * p.nspec; }

/// W3SIN4 (w3src4md.F90:423-1003) for one point. a (NSPEC), cg (NK), kk(ik) = K(1+(IK-1)NTH) is
/// kk[(ik-1)*kstride]; s, d (NSPEC) out; llws (NSPEC) out; tauwx..tauwny in/out (only thread
/// role 0 writes them, read them after the call's final sync). eb (NK) is work.
WWB_PN void sin4(const Cta& cta, const st4::Params& p, const Fields& f, const float* a,
                 const float* cg, const float* kk, int kstride, float u, float ustar, float drat,
                 float as, float usdir, float z0, float* tauwx, float* tauwy, float* tauwnx,
                 float* tauwny, float* s, float* d, int* llws, float* dstab, float* eb,
                 Sin4Sh& sh) {
  const int nk = p.nk, nth = p.nth, nspec = p.nspec;
  // The per-IK factors of the stress scan that do not depend on the running stress (:721-738),
  // formed in parallel: ZCN, CM, CONST2, CNST, SWELLCOEFV, SWELLCOEFT.
  float* const zcn_k = eb + nk;
  float* const cm_k = eb + 2 * nk;
  float* const const2_k = eb + 3 * nk;
  float* const cnst_k = eb + 4 * nk;
  float* const swv_k = eb + 5 * nk;
  float* const swt_k = eb + 6 * nk;
  // 1. Preparations (:600-675).
  PFOR(i, 3 * nspec) dstab[i] = 0.0f;
  {
    const float const0 = (p.bbeta / kKappa2) * drat;
    PFOR(ik0, nk) {
      float e = 0.0f;
      for (int ith = 0; ith < nth; ++ith) e = e + a[ith + ik0 * nth];
      eb[ik0] = e;
      const int ik = ik0 + 1;
      const int is0 = 1 + (ik - 1) * nth;
      const float kis = kk[(ik - 1) * kstride];
      const float sig2is = f.sig2[is0 - 1];
      cm_k[ik0] = kis / sig2is;
      const2_k[ik0] = f.dden2[is0 - 1] / cg[ik - 1] * kGrav / (f.sig[ik] / kis * drat);
      cnst_k[ik0] = sig2is * const0;
      zcn_k[ik0] = dm::logf(kis * z0);
      swv_k[ik0] = -(p.sswellf[4] * drat * 2.0f * kis * sqrt_f(kTwoNuAir * sig2is));
      swt_k[ik0] = -(drat * p.sswellf[0] * 16.0f * (sig2is * sig2is) / kGrav);
    }
    if (p.sintailpar[0] < 0.5f) {
      // The analytic tail's terms that depend on J only (:886-917).
      const float signk = f.sig[nk];
      const float zinf = dm::logf(signk * signk / kGrav);
      const float dely = (kLogTpiOver005 - zinf) / static_cast<float>(kJtot);
      PFOR(j0, kJtot) {
        const float y = dm::expf(zinf + static_cast<float>(j0) * dely);
        const float ykm = (y / kKm);
        const float ykm2 = ykm * ykm;
        const float tensk = 1.0f + ykm2;
        sh.tail[0][j0] = y;
        sh.tail[1][j0] = ykm;
        sh.tail[2][j0] = sqrt_f(kGrav * tensk / y);
        sh.tail[3][j0] = 0.5f * (3.0f * ykm2 + 1.0f) * sqrt_f(kGrav / (y * tensk));
        sh.tail[6][j0] = kGrav * z0 / (sh.tail[2][j0] * sh.tail[2][j0]);
        if (p.sintailpar[2] > 0.0f) {
          const float ykm1 = (ykm - 1.0f);
          sh.tail[4][j0] = dm::expf(-0.25f * (ykm1 * ykm1));
          sh.tail[5][j0] = dm::tanhf((y - 20.0f) / 5.0f);
        }
      }
    }
  }
  cta.sync();
  if (cta.role(0)) {
    const float const1 = p.bbeta / kKappa2;
    const float const0 = const1 * drat;
    const float z0visc = kZ0viscNum / max_r(ustar, 0.0001f);
    const float z0noz = max_r(z0visc, p.zz0rat * z0);
    float uorb = 0.0f, aorb = 0.0f;
    for (int ik = 1; ik <= nk; ++ik) {
      const float sigk = f.sig[ik];
      uorb = uorb + eb[ik - 1] * (sigk * sigk) * f.dden[ik - 1] / cg[ik - 1];
      aorb = aorb + eb[ik - 1] * f.dden[ik - 1] / cg[ik - 1];
    }
    uorb = 2.0f * sqrt_f(uorb);
    const float aorb1 = 2.0f * dm::powf(aorb, 1.0f - 0.5f * p.sswellf[5]);
    const float re = 4.0f * uorb * aorb1 / kNuAir;
    float pturb, pvisc;
    if (p.sswellf[3] > 0.0f) {
      if (p.sswellf[6] > 0.0f) {
        const float smooth = 0.5f * dm::tanhf((re - p.sswellf[3]) / p.sswellf[6]);
        pturb = (0.5f + smooth);
        pvisc = (0.5f - smooth);
      } else if (re <= p.sswellf[3]) {
        pturb = 0.0f;
        pvisc = 1.0f;
      } else {
        pturb = 1.0f;
        pvisc = 0.0f;
      }
    } else {
      pturb = 1.0f;
      pvisc = 1.0f;
    }
    float fw, fu, fud;
    if (p.sswellf[1] == 0.0f) {
      fw = fabs_f(p.sswellf[2]);
      fu = 0.0f;
      fud = 0.0f;
    } else {
      fu = fabs_f(p.sswellf[2]);
      fud = p.sswellf[1];
      aorb = 2.0f * sqrt_f(aorb);
      const float xi = (dm::log10f(max_r(aorb / z0noz, 3.0f)) - kAbMin) / p.delab;
      const int ind = min_i(st4::kSizeFwTable - 1, fint(xi));
      const float deli1 = min_r(1.0f, xi - static_cast<float>(ind));
      const float deli2 = 1.0f - deli1;
      fw = f.fwtable[ind] * deli2 + f.fwtable[ind + 1] * deli1;
    }
    float ustarsigma = 0.0f;
    if (p.stab3) {
      float usigma;
      if (isnan_f(as)) {
        usigma = 0.0f;
      } else {
        usigma = max_r(0.0f, -0.025f * as);
      }
      ustarsigma = (1.0f + u / (10.0f + u)) * usigma;
    }
    sh.const1 = const1;
    sh.const0 = const0;
    sh.uorb = uorb;
    sh.pturb = pturb;
    sh.pvisc = pvisc;
    sh.fw = fw;
    sh.fu = fu;
    sh.fud = fud;
    sh.ustarsigma = ustarsigma;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 2; ++j) sh.ss[i][j] = sh.sn[i][j] = 0.0f;
  }
  cta.sync();

  // 2. The stress scan over IK (:696-797). The threads of the first nth (or all, if fewer)
  //    carry identical copies of the running stress sums: each computes the per-IK scalars,
  //    the terms of its directions, and then adds all directions' terms in ITH order.
  const int nscan = nth < cta.nthr ? nth : cta.nthr;
  const bool scan = cta.tid < nscan;
  const float uorb = sh.uorb, pturb = sh.pturb, pvisc = sh.pvisc,
              fw = sh.fw, fu = sh.fu, fud = sh.fud, ustarsigma = sh.ustarsigma;
  float ust = ustar, taux = 0.0f, tauy = 0.0f, cosu = 0.0f, sinu = 0.0f, ustp = 0.0f,
        usdirp = 0.0f;
  const int istab_first = p.stab3 ? 1 : 3, istab_last = p.stab3 ? 2 : 3;
  int parity = 0;
  for (int istab = istab_first; istab <= istab_last; ++istab) {
    if (istab == 1) ust = ustar * (1.0f - ustarsigma);
    if (istab == 2) ust = ustar * (1.0f + ustarsigma);
    float cu, su;
    dm::sincosf(usdir, &su, &cu);
    taux = (ust * ust) * cu;
    tauy = (ust * ust) * su;
    // The running sums of this pass (STRESSSTAB, STRESSSTABN of ISTAB), in registers.
    float ssi0 = 0.0f, ssi1 = 0.0f, sni0 = 0.0f, sni1 = 0.0f;
    for (int ik = 1; ik <= nk; ++ik, parity ^= 1) {
      if (scan) {
        const float taupx = taux - fabs_f(p.ttauwshelter) * ssi0;
        const float taupy = tauy - fabs_f(p.ttauwshelter) * ssi1;
        ustp = min_r(dm::powf((taupx * taupx + taupy * taupy), 0.25f), max_r(ust, 0.3f));
        usdirp = dm::atan2f(taupy, taupx);
        dm::sincosf(usdirp, &sinu, &cosu);
        const int is0 = 1 + (ik - 1) * nth;
        const float sig2is = f.sig2[is0 - 1];
        const float cm = cm_k[ik - 1];
        const float ucn = ustp * cm + p.zzalp;
        const float const2 = const2_k[ik - 1];
        const float cnst = cnst_k[ik - 1];
        const float zcn = zcn_k[ik - 1];
        const float swellcoefv = swv_k[ik - 1];
        const float swellcoeft = swt_k[ik - 1];
        for (int ith = cta.tid; ith < nth; ith += nscan) {
          const int is = ith + 1 + (ik - 1) * nth;
          const float ecos = f.ecos[is - 1], esin = f.esin[is - 1];
          const float coswind = (ecos * cosu + esin * sinu);
          float dst;
          int lw;
          if (coswind > 0.01f) {
            const float x = coswind * ucn;
            const float zarg = kKappa / x;
            const float zlog = zcn + zarg;
            if (zlog < 0.0f) {
              const float zlog2 = zlog * zlog;
              dst = cnst * dm::expf(zlog) * (zlog2 * zlog2) * ucn * ucn *
                    dm::powf(coswind, p.ssinthp);
              lw = 1;
            } else {
              dst = 0.0f;
              lw = 0;
            }
            if (28.0f * cm * ustar * coswind >= 1.0f) lw = 1;
          } else {
            dst = 0.0f;
            lw = 0;
          }
          if ((p.sswellf[0] != 0.0f && dst < 1E-7f * sig2is) || p.sswellf[2] > 0.0f) {
            const float dvisc = swellcoefv;
            const float dturb = swellcoeft * (fw * uorb + (fu + fud * coswind) * ustp);
            dst = dst + pturb * dturb + pvisc * dvisc;
          }
          dstab[(istab - 1) * nspec + (is - 1)] = dst;
          llws[is - 1] = lw;
          const float temp2 = const2 * dst * a[is - 1];
          sh.term[parity][0][ith] = temp2 * ecos;
          sh.term[parity][1][ith] = temp2 * esin;
          sh.term[parity][2][ith] = dst < 0.0f ? 1.0f : 0.0f;
        }
      }
      cta.sync();
      if (scan) {
WWB_UNROLL(4)
        for (int ith = 0; ith < nth; ++ith) {
          const float t0 = sh.term[parity][0][ith], t1 = sh.term[parity][1][ith];
          if (sh.term[parity][2][ith] != 0.0f) {
            sni0 = sni0 + t0;
            sni1 = sni1 + t1;
          } else {
            ssi0 = ssi0 + t0;
            ssi1 = ssi1 + t1;
          }
        }
      }
    }
    if (cta.role(0)) {
      sh.ss[istab - 1][0] = ssi0;
      sh.ss[istab - 1][1] = ssi1;
      sh.sn[istab - 1][0] = sni0;
      sh.sn[istab - 1][1] = sni1;
    }
  }
  if (cta.role(0)) {
    sh.ust = ust;
    sh.taux = taux;
    sh.tauy = tauy;
    sh.cosu = cosu;
    sh.sinu = sinu;
    sh.ustp = ustp;
    sh.usdirp = usdirp;
  }
  cta.sync();

  // 3. D, S, the tail stress and the stress limit (:799-976).
  if (!p.stab3) {
    PFOR(i, nspec) d[i] = dstab[2 * nspec + i];
  } else {
    PFOR(i, nspec) d[i] = 0.5f * (dstab[i] + dstab[nspec + i]);
  }
  PFOR(i, nspec) s[i] = (!p.stab3 ? dstab[2 * nspec + i] : 0.5f * (dstab[i] + dstab[nspec + i])) * a[i];
  if (cta.role(0)) {
    float xstress, ystress, twnx, twny;
    if (!p.stab3) {
      xstress = sh.ss[2][0];
      ystress = sh.ss[2][1];
      twnx = sh.sn[2][0];
      twny = sh.sn[2][1];
    } else {
      xstress = 0.5f * (sh.ss[0][0] + sh.ss[1][0]);
      ystress = 0.5f * (sh.ss[0][1] + sh.ss[1][1]);
      twnx = 0.5f * (sh.sn[0][0] + sh.sn[1][0]);
      twny = 0.5f * (sh.sn[0][1] + sh.sn[1][1]);
    }
    *tauwnx = twnx;
    *tauwny = twny;
    float ustl, usdirpl;
    {
      const float taupx = sh.taux - fabs_f(p.ttauwshelter) * xstress;
      const float taupy = sh.tauy - fabs_f(p.ttauwshelter) * ystress;
      ustl = dm::powf((taupx * taupx + taupy * taupy), 0.25f);
      usdirpl = dm::atan2f(taupy, taupx);
    }
    const float ust3 = ustl;
    float c0;
    {
      const float signk = f.sig[nk];
      const float s2 = signk * signk;
      const float s5 = s2 * (s2 * signk);
      c0 = p.dth * s5 / kGrav2Tpi * kTpi * signk / cg[nk - 1];
    }
    float temp = 0.0f;
    for (int ith = 1; ith <= nth; ++ith) {
      const int is = ith + (nk - 1) * nth;
      const float coswind = (f.ecos[is - 1] * sh.cosu + f.esin[is - 1] * sh.sinu);
      const float cp = (max_r(coswind, 0.0f));
      temp = temp + a[is - 1] * (cp * (cp * cp));
    }
    const float levtail0 = c0 * temp;
    float tauhf;
    if (p.sintailpar[0] < 0.5f) {
      float ustr = ust3;
      const float signk = f.sig[nk];
      const float zinf = dm::logf(signk * signk / kGrav);
      const float dely = (kLogTpiOver005 - zinf) / static_cast<float>(kJtot);
      float taur = ust3 * ust3;
      float tau1 = 0.0f;
      for (int j = 1; j <= kJtot; ++j) {
        const float w = (j == 1 || j == kJtot) ? 0.5f : 1.0f;
        const float cm = sh.tail[2][j - 1];
        const float cgtail = sh.tail[3][j - 1];
        const float zx = ustr / cm + p.zzalp;
        const float zarg = min_r(kKappa / zx, 20.0f);
        const float zmu = min_r(sh.tail[6][j - 1] * dm::expf(zarg), 1.0f);
        const float zlog = min_r(dm::logf(zmu), 0.0f);
        const float zlog2 = zlog * zlog;
        const float zbeta = sh.const1 * zmu * (zlog2 * zlog2);
        float levtail;
        if (p.sintailpar[2] > 0.0f) {
          float alpham;
          if (ustr < cm) {
            alpham = max_r(0.0f, 0.01f * (1.0f + dm::logf(ustr / cm)));
          } else {
            alpham = 0.01f * (1.0f + 3.0f * dm::logf(ustr / cm));
          }
          const float fm = sh.tail[4][j - 1];
          const float alphat = alpham * (kCmm / cm) * fm;
          const float th = sh.tail[5][j - 1];
          levtail = levtail0 * 0.5f * (1.0f - th) + p.sintailpar[2] * 0.5f * (1.0f + th) * alphat;
        } else {
          levtail = levtail0;
        }
        tau1 = tau1 + w * zbeta * (ustr * ustr) * levtail * dely * cgtail / cm;
        taur = taur - w * p.sintailpar[1] * (ustr * ustr) * zbeta * levtail * dely * cgtail / cm;
        ustr = sqrt_f(max_r(taur, 0.0f));
      }
      tauhf = tau1;
    } else {
      const float xi = ust3 / p.delust;
      const int ind = max_i(1, min_i(st4::kIustar - 1, fint(xi)));
      const float deli1 = max_r(min_r(1.0f, xi - static_cast<float>(ind)), 0.0f);
      const float deli2 = 1.0f - deli1;
      const float ustm = max_r(ust3, 0.00001f);
      const float xj = max_r(0.0f, (kGrav * z0 / (ustm * ustm) - p.aalpha) / p.delalp);
      const int j = max_i(1, min_i(st4::kIalpha - 1, fint(xj)));
      const float delj1 = max_r(0.0f, min_r(1.0f, xj - static_cast<float>(j)));
      const float delj2 = 1.0f - delj1;
      float tau1;
      if (p.ttauwshelter > 0.0f) {
        const float xk = levtail0 / p.deltail;
        const int i = min_i(st4::kIlevTail - 1, fint(xk));
        const float delk1 = min_r(1.0f, xk - static_cast<float>(i));
        const float delk2 = 1.0f - delk1;
        tau1 = ((f.tauhft2_at(ind, j, i) * deli2 + f.tauhft2_at(ind + 1, j, i) * deli1) * delj2 +
                (f.tauhft2_at(ind, j + 1, i) * deli2 + f.tauhft2_at(ind + 1, j + 1, i) * deli1) *
                    delj1) * delk2 +
               ((f.tauhft2_at(ind, j, i + 1) * deli2 + f.tauhft2_at(ind + 1, j, i + 1) * deli1) *
                    delj2 +
                (f.tauhft2_at(ind, j + 1, i + 1) * deli2 +
                 f.tauhft2_at(ind + 1, j + 1, i + 1) * deli1) *
                    delj1) *
                   delk1;
      } else {
        tau1 = (f.tauhft_at(ind, j) * deli2 + f.tauhft_at(ind + 1, j) * deli1) * delj2 +
               (f.tauhft_at(ind, j + 1) * deli2 + f.tauhft_at(ind + 1, j + 1) * deli1) * delj1;
      }
      tauhf = levtail0 * (ust3 * ust3) * tau1;
    }
    float cp, sp;
    dm::sincosf(usdirpl, &sp, &cp);
    float twx = xstress + tauhf * cp;
    float twy = ystress + tauhf * sp;
    const float tauw = sqrt_f(twx * twx + twy * twy);
    const float ust2b = max_r(ustar, kEps2);
    const float ust2 = ust2b * ust2b;
    const float tauwb = min_r(tauw, max_r(ust2 - kEps1, kEps2Sq));
    if (tauwb < tauw) {
      twx = twx * tauwb / tauw;
      twy = twy * tauwb / tauw;
    }
    *tauwx = twx;
    *tauwy = twy;
  }
  cta.sync();
}

// ================================================================================ CALC_USTAR
/// CALC_USTAR (w3src4md.F90:1849-2011), serial. MIN/MAX as (b < a) ? b : a (b > a) ? b : a.
WWB_PN void calc_ustar(const st4::Params& p, const Fields& f, float windspeed, float tauw,
                       float* ustar_io, float* z0, float* charn) {
  auto fmin2 = [](float a, float b) { return (b < a) ? b : a; };
  auto fmax2 = [](float a, float b) { return (b > a) ? b : a; };
  auto imin2 = [](int a, int b) { return (b < a) ? b : a; };
  constexpr int kNiter = 10;
  constexpr float kXm = 0.50f, kE1 = 0.00001f;
  float chath = p.aalpha;
  float ustar = *ustar_io;
  float ust = 0.0f;
  if (p.sintailpar[0] > 0.5f) {
    const float tauw_local = fmax2(fmin2(tauw, 2.2361f), 0.0f);
    const float xi = sqrt_f(tauw_local) / p.deltauw;
    const int ind = imin2(st4::kItauMax - 1, fint(xi));
    const float deli1 = fmin2(1.0f, xi - static_cast<float>(ind));
    const float deli2 = 1.0f - deli1;
    const float xj = windspeed / p.delu;
    const int j = imin2(st4::kJuMax - 1, fint(xj));
    const float delj1 = fmin2(1.0f, xj - static_cast<float>(j));
    const float delj2 = 1.0f - delj1;
    ustar = (f.taut_at(ind, j) * deli2 + f.taut_at(ind + 1, j) * deli1) * delj2 +
            (f.taut_at(ind, j + 1) * deli2 + f.taut_at(ind + 1, j + 1) * deli1) * delj1;
  } else {
    float xmin;
    if (p.capchnk[0] == 1.0f) {
      chath = p.capchnk[1] + 0.5f * (p.capchnk[2] - p.capchnk[1]) *
                                 (1.0f - dm::tanhf((windspeed - p.capchnk[3]) / p.capchnk[4]));
      xmin = 0.15f * (p.capchnk[2] - chath);
    } else {
      xmin = 0.0f;
    }
    const float tauw_local = tauw;
    const float wcd = sqrt_f(0.0012875f);
    const float ustold = windspeed * wcd;
    float tauold = fmax2(ustold * ustold, tauw_local + kE1);
    constexpr float kZnuNum = 0.11f * kNuAir;
    constexpr float kXm1 = kXm + 1.0f;
    for (int iter = 1; iter <= kNiter; ++iter) {
      const float x = fmax2(tauw_local / tauold, xmin);
      ust = sqrt_f(tauold);
      float zz00 = chath * tauold / kGrav;
      if (p.zz0max != 0.0f) zz00 = fmin2(zz00, p.zz0max);
      const float omx = 1.0f - x;
      float zz0 = zz00 / dm::powf(omx, kXm);
      const float znu = kZnuNum / fmax2(ust, 1E-6f);
      zz0 = p.sintailpar[4] * znu + zz0;
      const float lg = dm::logf(p.zzwnd / zz0);
      const float fval = ust - kKappa * windspeed / lg;
      const float delf =
          1.0f - kKappa * windspeed / (lg * lg) * 2.0f / ust * (1.0f - kXm1 * x) / omx;
      ust = ust - fval / delf;
      tauold = fmax2(ust * ust, tauw_local + kE1);
    }
    ustar = ust;
  }
  if (ustar > 0.001f) {
    const float sqrtcdm1 = fmin2(windspeed / ustar, 100.0f);
    *z0 = p.zzwnd * dm::expf(-kKappa * sqrtcdm1);
    *charn = kGrav * *z0 / (ustar * ustar);
  } else {
    if (ustar > 0.0f) {
      const float sqrtcdm1 = fmin2(windspeed / ustar, 100.0f);
      *z0 = p.zzwnd * dm::expf(-kKappa * sqrtcdm1);
    } else {
      *z0 = chath * 0.001f * 0.001f / kGrav;
    }
    *charn = chath;
  }
  if (p.capchnk[0] == 1.0f) {
    *charn = fmin2(0.09f, *charn);
    if (*charn < chath) *charn = chath;
  }
  *ustar_io = ustar;
}

// ===================================================================================== W3SPR4
/// The W3SPR4 outputs (all INOUT at the boundary).
struct Spr4Out {
  float ustar, usdir, emean, fmean, fmean1, wnmean, amax, cd, z0, charn, fmeanws, dlwmean;
};

/// Reals of W3SPR4 work: EB, EB2, the two powers and SIGFAC (NK each) and three chain results;
/// terms holds 2 x NSPEC more (the ELCS / ELSN terms).
WWB_PD int spr4_work_reals(const st4::Params& p) { return 5 * p.nk + 4; }
WWB_PD int spr4_terms_reals(const st4::Params& p) { return 2 * p.nspec; }

/// W3SPR4 (w3src4md.F90:142-384) for one point. a, llws (NSPEC); cg, wn (NK); o is read (ustar
/// in) and written by role 0. The libmvec powers of :316 and :317 use scalar powf in every lane.
/// ELCS and ELSN are one running sum each over IK then ITH, AMAX one running MAX: their terms
/// are formed in parallel, then each chain runs on its own thread in the reference's order.
WWB_PN void spr4(const Cta& cta, const st4::Params& p, const Fields& f, const float* a,
                 const float* cg, const float* wn, float u, float udir, float tauwx,
                 float tauwy, const int* llws, Spr4Out& o, float* work, float* terms) {
  const int nk = p.nk, nth = p.nth, nspec = p.nspec;
  float* const eb = work;
  float* const eb2 = work + nk;
  float* const pwsig = work + 2 * nk;
  float* const pwwn = work + 3 * nk;
  float* const sigfac = work + 4 * nk;
  float* const chains = work + 5 * nk;  // ELCS, ELSN, AMAX
  float* const tc = terms;
  float* const ts = terms + nspec;
  // Per-IK direction sums (independent over IK), the two powers and SIGFAC.
  PFOR(ik0, nk) {
    const int ik = ik0 + 1;
    float ebk = 0.0f, eb2k = 0.0f;
    for (int ith = 1; ith <= nth; ++ith) {
      const int is = ith + (ik - 1) * nth;
      const float aa = a[(ik - 1) * nth + ith - 1];
      ebk = ebk + aa;
      if (llws[is - 1] != 0) eb2k = eb2k + aa;
    }
    eb[ik0] = ebk;
    eb2[ik0] = eb2k;
    pwsig[ik0] = dm::powf(f.sig[ik], 2.0f * p.wwnmeanptail);
    pwwn[ik0] = dm::powf(wn[ik0], p.wwnmeanp);
    sigfac[ik0] = dm::powf(f.sig[ik], p.ssdsc[11]) * f.dden[ik - 1] / cg[ik - 1];
  }
  cta.sync();
  PFOR(is0, nspec) {
    const float aa = a[is0];
    const float sf = sigfac[is0 / nth];
    tc[is0] = aa * f.ecos[is0] * sf;
    ts[is0] = aa * f.esin[is0] * sf;
  }
  cta.sync();
  if (cta.role(0)) {
    float v = 0.0f;
WWB_UNROLL(8)
    for (int i = 0; i < nspec; ++i) v = v + tc[i];
    chains[0] = v;
  }
  if (cta.role(1)) {
    float v = 0.0f;
WWB_UNROLL(8)
    for (int i = 0; i < nspec; ++i) v = v + ts[i];
    chains[1] = v;
  }
  if (cta.role(2)) {
    float v = 0.0f;
WWB_UNROLL(8)
    for (int i = 0; i < nspec; ++i) v = max_r(v, a[i]);
    chains[2] = v;
  }
  cta.sync();
  if (cta.role(0)) {
    const float eps = 1.E-7f;
    float ustar = max_r(0.0001f, o.ustar);
    const float dlwmean = dm::atan2f(chains[1], chains[0]);
    const float amax = chains[2];
    float emean = 0.0f, fmean = 0.0f, fmean1 = 0.0f, wnmean = 0.0f, emeanws = 0.0f,
          fmeanws = 0.0f;
    for (int ik = 1; ik <= nk; ++ik) {
      const float ebk = eb[ik - 1] * f.dden[ik - 1] / cg[ik - 1];
      const float eb2k = eb2[ik - 1] * f.dden[ik - 1] / cg[ik - 1];
      eb[ik - 1] = ebk;
      eb2[ik - 1] = eb2k;
      emean = emean + ebk;
      fmean = fmean + ebk / f.sig[ik];
      fmean1 = fmean1 + ebk * pwsig[ik - 1];
      wnmean = wnmean + ebk * pwwn[ik - 1];
      emeanws = emeanws + eb2k;
      fmeanws = fmeanws + eb2k * pwsig[ik - 1];
    }
    float eband = eb[nk - 1] / f.dden[nk - 1];
    emean = emean + eband * p.fte;
    fmean = fmean + eband * p.ftf;
    fmean1 = fmean1 + eband * p.sstxftftail;
    wnmean = wnmean + eband * p.sstxftwn;
    eband = eb2[nk - 1] / f.dden[nk - 1];
    emeanws = emeanws + eband * p.fte;
    fmeanws = fmeanws + eband * p.sstxftftail;
    fmean = kTpiInv * emean / max_r(eps, fmean);
    if (fmean1 < eps) {
      fmean1 = kTpiInv * f.sig[nk];
    } else {
      fmean1 = kTpiInv * dm::powf(max_r(eps, fmean1) / max_r(eps, emean),
                                  1.0f / (2.0f * p.wwnmeanptail));
    }
    wnmean = dm::powf(max_r(eps, wnmean) / max_r(eps, emean), 1.0f / p.wwnmeanp);
    if (fmeanws < eps || emeanws < eps) {
      fmeanws = kTpiInv * f.sig[nk];
    } else {
      fmeanws = kTpiInv * dm::powf(max_r(eps, fmeanws) / max_r(eps, emeanws),
                                   1.0f / (2.0f * p.wwnmeanptail));
    }
    const float tauw = sqrt_f(tauwx * tauwx + tauwy * tauwy);
    float z0 = o.z0, charn = o.charn;
    calc_ustar(p, f, u, tauw, &ustar, &z0, &charn);
    const float unz = max_r(0.01f, u);
    const float r = ustar / unz;
    o.ustar = ustar;
    o.usdir = udir;
    o.emean = emean;
    o.fmean = fmean;
    o.fmean1 = fmean1;
    o.wnmean = wnmean;
    o.amax = amax;
    o.cd = r * r;
    o.z0 = z0;
    o.charn = charn;
    o.fmeanws = fmeanws;
    o.dlwmean = dlwmean;
  }
  cta.sync();
}

// ===================================================================================== W3SDS4
constexpr float kTwoPiSq = 2.0f * (kPi * kPi);
constexpr float kGrav2 = kGrav * kGrav;
constexpr float kTwoPi = 2.0f * kPi;
constexpr float kTstrFac = (0.8f * 2.0f) * kPi;
constexpr float kTmaxFac = (5.0f * 2.0f) * kPi;
constexpr float kDkhs = 2.0f / static_cast<float>(st4::kNkhs);
constexpr float kLogFacKd1 = 9.9503211677074432373046875e-3f;  // LOG(1.01), folded
constexpr int kFacKd2 = 1000;

/// FLOOR(x) as the -O3 build computes it (st4_sds4.hpp:54-58).
WWB_PD int ffloor(float x) {
  const int i = fint(x);
  return static_cast<float>(i) <= x ? i : static_cast<int>(static_cast<unsigned>(i) - 1u);
}

/// Reals and ints of W3SDS4 work: work holds the NK arrays and MSSSUM(NK,5) (18 NK), work2
/// BTH, PB, PB2 (3 NSPEC).
WWB_PD int sds4_work_reals(const st4::Params& p) { return 18 * p.nk; }
WWB_PD int sds4_work2_reals(const st4::Params& p) { return 3 * p.nspec; }
WWB_PD int sds4_work_ints(const st4::Params& p) { return 2 * p.nk; }

struct Sds4Sh {
  float facturb;
  int dikcumul, ik1, nkl;
};

/// W3SDS4 (w3src4md.F90:2043-2659) for one point. a, srhs, ddiag, brlambda (NSPEC); kk, cg (NK);
/// whitecap (4) in/out. The libmvec loops (:2315, :2500, :2509) use scalar powf/expf per lane.
WWB_PN void sds4(const Cta& cta, const st4::Params& p, const Fields& f, const float* a,
                 const float* kk, const float* cg, float ustar, float usdir, float depth,
                 float dair, float dlwmean, int flogrd57, int flogrd58, float* srhs,
                 float* ddiag, float* brlambda, float* whitecap, float* work, float* work2,
                 int* iwork, Sds4Sh& sh) {
  const int nk = p.nk, nth = p.nth, nspec = p.nspec;
  const float* ssdsc = p.ssdsc;
  const float zero = 0.0f, one = 1.0f;
  float* const coef4 = work;
  float* const coef5 = coef4 + nk;
  float* const s1 = coef5 + nk;
  float* const e1 = s1 + nk;
  float* const dk = e1 + nk;
  float* const hs = dk + nk;
  float* const kbar = hs + nk;
  float* const dck = kbar + nk;
  float* const efdf = dck + nk;
  float* const bth0 = efdf + nk;
  float* const qb = bth0 + nk;
  float* const s2 = qb + nk;
  float* const brm12 = s2 + nk;
  float* const msssum = brm12 + nk;  // MSSSUM(IK,J) = msssum[(J-1)*nk + IK-1]
  float* const bth = work2;
  float* const pb = bth + nspec;
  float* const pb2 = pb + nspec;
  int* const ntimes = iwork;
  int* const iksup = iwork + nk;
  auto MSS = [&](int ik, int j) -> float& { return msssum[(j - 1) * nk + (ik - 1)]; };

  // 0. Pre-initialisation (:2203-2213) and section 1 (:2217-2224).
  PFOR(i, nk) {
    s1[i] = e1[i] = dk[i] = hs[i] = kbar[i] = dck[i] = efdf[i] = bth0[i] = qb[i] = s2[i] =
        brm12[i] = zero;
    ntimes[i] = iksup[i] = 0;
  }
  PFOR(i, nspec) bth[i] = ddiag[i] = srhs[i] = pb[i] = pb2[i] = zero;
  PFOR(i, 5 * nk) msssum[i] = zero;
  if (cta.role(0)) {
    sh.facturb = (((ssdsc[4] * (ustar * ustar)) / kGrav) * dair) / kDwat;
    sh.dikcumul = nint(p.ssdsbrf1 / (p.xfr - one));
    sh.ik1 = p.ig1 ? nint(p.igpars5) + 1 : 1;
  }
  cta.sync();
  const int ik1 = sh.ik1;

  // 1.b Mean-square slope (:2228-2254): per-IK direction sums, then the running sums over IK.
  const bool mss = ssdsc[7] > zero || ssdsc[10] > zero || ssdsc[17] > zero;
  if (mss) {
    // coef4/coef5/dk are free here: per-IK MSSP, MSSPC2, MSSPS2.
    PFOR(ik0, nk) {
      const int ik = ik0 + 1;
      float mssp = zero, msspc2 = zero, mssps2 = zero;
      const float kp = dm::powf(kk[ik - 1], ssdsc[19]);
      for (int ith = 1; ith <= nth; ++ith) {
        const int is = ith + (ik - 1) * nth;
        const float msslong = ((kp * a[is - 1]) * f.dden[ik - 1]) / cg[ik - 1];
        msspc2 = msspc2 + msslong * f.ecos[ith - 1];
        mssps2 = mssps2 + msslong * f.esin[ith - 1];
        mssp = mssp + msslong;
      }
      coef4[ik0] = mssp;
      coef5[ik0] = msspc2;
      dk[ik0] = mssps2;
    }
    cta.sync();
    PFOR(i0, nk) {
      float m1 = zero, m3 = zero, m4 = zero;
      for (int ik = 0; ik <= i0; ++ik) {
        m1 = m1 + coef4[ik];
        m3 = m3 + coef5[ik];
        m4 = m4 + dk[ik];
      }
      MSS(i0 + 1, 1) = m1;
      MSS(i0 + 1, 3) = m3;
      MSS(i0 + 1, 4) = m4;
      float mssd = dm::atan2f(m4, m3);
      if (mssd < zero) mssd = mssd + kPi;
      MSS(i0 + 1, 2) = mssd;
    }
    cta.sync();
    PFOR(i, nk) coef4[i] = coef5[i] = dk[i] = zero;
    cta.sync();
  }

  const int sdscase = nint(ssdsc[0]);
  if (sdscase == 1) {
    // 2.a.1 Saturation (:2262-2290).
    const float dth = p.dth;
    PFOR(ik0, nk) {
      const int ik = ik0 + 1;
      if (ik >= ik1) {
        const float kx = kk[ik - 1];
        const float facsat = (f.sig[ik] * ((kx * kx) * kx)) * dth;
        const int is0 = (ik - 1) * nth;
        float asum = zero;
        for (int ith = 1; ith <= nth; ++ith) asum = asum + a[is0 + ith - 1];
        bth0[ik - 1] = asum * facsat;
      }
    }
    cta.sync();
    if (p.ssdsdth >= 180.0f) {
      PFOR(i, nspec) {
        const int ik = i / nth + 1;
        if (ik >= ik1) bth[i] = bth0[ik - 1];
      }
    } else {
      PFOR(i, nspec) {
        const int ik = i / nth + 1, ith0 = i - (ik - 1) * nth;
        if (ik >= ik1) {
          const int is0 = (ik - 1) * nth;
          float v = zero;
          for (int j = 0; j < f.nsat; ++j)
            v = v + f.satw_t[ith0 + j * f.sat_ld] * a[is0 + f.sati_t[ith0 + j * f.sat_ld] - 1];
          const float kx = kk[ik - 1];
          const float facsat = (f.sig[ik] * ((kx * kx) * kx)) * dth;
          bth[i] = v * facsat;
        }
      }
      cta.sync();
      // MAXVAL as gfortran lowers it: the first element >= -Inf, then strictly greater.
      PFOR(ik0, nk) {
        const int ik = ik0 + 1;
        if (ik >= ik1) {
          const int is0 = (ik - 1) * nth;
          float lim = -dm::asfloat(0x7f800000u);
          int i = is0;
          bool found = false;
          for (; i < is0 + nth; ++i) {
            if (bth[i] >= lim) {
              lim = bth[i];
              ++i;
              found = true;
              break;
            }
          }
          if (!found) lim = dm::asfloat(0x7fc00000u);
          for (; i < is0 + nth; ++i)
            if (bth[i] > lim) lim = bth[i];
          bth0[ik - 1] = lim;
        }
      }
    }
    cta.sync();
    // 2.a.2 Spontaneous breaking (:2291-2331).
    const float epsr = sqrt_f(p.ssdsbr);
    PFOR(i, nspec) {
      const int ik = i / nth + 1;
      if (ik >= ik1) {
        float miche;
        if (p.ssdsbm[0] == one) {
          miche = one;
        } else {
          const float x = dm::tanhf(min_r(kk[ik - 1] * depth, 10.0f));
          const float t =
              x * (p.ssdsbm[1] + x * (p.ssdsbm[2] + x * (p.ssdsbm[3] + x * p.ssdsbm[4])));
          miche = t * t;
        }
        const float coef1 = p.ssdsbr * miche;
        const float m = max_r(bth0[ik - 1] / coef1 - one, zero);
        const float sdiagiso = ((ssdsc[1] * f.sig[ik]) * ssdsc[5]) * (m * m);
        const float coef2 = ((ssdsc[1] * f.sig[ik]) * (one - ssdsc[5])) / (coef1 * coef1);
        ddiag[i] = sdiagiso + coef2 * dm::powf(max_r(bth[i] - coef1, zero), p.ssdsp);
      }
    }
    cta.sync();
    PFOR(i, nspec) {
      const float m = max_r(sqrt_f(bth[i]) - epsr, zero);
      float pbi = m * m;
      pbi = pbi * 28.16f;
      pb[i] = pbi;
      brlambda[i] = pbi / kTwoPiSq;
      srhs[i] = ddiag[i] * a[i];
    }
    cta.sync();
  } else if (sdscase == 2) {
    // 2.b Filipot et al. (:2338-2477).
    const float dth = p.dth;
    PFOR(i, nk) e1[i] = hs[i] = zero;
    PFOR(i, nspec) srhs[i] = ddiag[i] = pb2[i] = zero;
    cta.sync();
    PFOR(ik0, nk) {
      const int ik = ik0 + 1;
      if (ik >= ik1) {
        float e = zero;
        for (int ith = 1; ith <= nth; ++ith) {
          const int is = ith + (ik - 1) * nth;
          e = e + (a[is - 1] * f.sig[ik]) * dth;
        }
        e1[ik - 1] = e;
        dk[ik - 1] = f.dden[ik - 1] / ((dth * f.sig[ik]) * cg[ik - 1]);
      }
    }
    cta.sync();
    if (cta.role(0)) {
      int id = nint(depth);
      if (id > st4::kNdtab) id = st4::kNdtab;
      if (id < 1) id = 1;
      int nkl = 0;
      for (int i = 0; i < nk; ++i) hs[i] = efdf[i] = kbar[i] = zero;
      for (int ikl = 1; ikl <= nk; ++ikl) {
        iksup[ikl - 1] = f.iktab[(ikl - 1) + (id - 1) * f.iktab_ld];
        if (iksup[ikl - 1] <= nk) {
          float v = zero;
          for (int i = ikl; i <= iksup[ikl - 1] - 1; ++i) v = v + e1[i - 1] * dk[i - 1];
          efdf[ikl - 1] = v;
          if (efdf[ikl - 1] != zero) {
            float w = zero;
            for (int i = ikl; i <= iksup[ikl - 1] - 1; ++i) w = w + (kk[i - 1] * e1[i - 1]) * dk[i - 1];
            kbar[ikl - 1] = w / efdf[ikl - 1];
          } else {
            kbar[ikl - 1] = zero;
          }
          hs[ikl - 1] = 4.0f * sqrt_f(efdf[ikl - 1]);
          nkl = nkl + 1;
        }
      }
      for (int i = 0; i < nk; ++i) dck[i] = qb[i] = zero;
      for (int ikl = 1; ikl <= nkl; ++ikl) {
        const float kb = kbar[ikl - 1];
        if (hs[ikl - 1] != zero && kb != zero) {
          int ikd = fint(roundf(dm::logf(kb * depth) / kLogFacKd1) + static_cast<float>(kFacKd2));
          int ikhs = fint(one + roundf((kb * hs[ikl - 1]) / kDkhs));
          if (ikd > st4::kNkd) ikd = st4::kNkd;
          else if (ikd < 1) ikd = 1;
          if (ikhs > st4::kNkhs) ikhs = st4::kNkhs;
          else if (ikhs < 1) ikhs = 1;
          dck[ikl - 1] = (dm::powf(kb, -2.5f) * (kb / kTwoPi)) *
                         f.dcki[(ikhs - 1) + (ikd - 1) * st4::kNkhs];
          qb[ikl - 1] = f.qbi[(ikhs - 1) + (ikd - 1) * st4::kNkhs];
        } else {
          dck[ikl - 1] = zero;
          qb[ikl - 1] = zero;
        }
      }
      for (int i = 0; i < nk; ++i) {
        s1[i] = s2[i] = zero;
        ntimes[i] = 0;
      }
      for (int ikl = 1; ikl <= nkl; ++ikl) {
        if (efdf[ikl - 1] > zero) {
          for (int i = ikl; i <= iksup[ikl - 1]; ++i)
            s1[i - 1] = s1[i - 1] + (dck[ikl - 1] * e1[i - 1]) / efdf[ikl - 1];
          for (int i = ikl; i <= iksup[ikl - 1]; ++i)
            s2[i - 1] = s2[i - 1] + (qb[ikl - 1] * e1[i - 1]) / efdf[ikl - 1];
          for (int i = ikl; i <= iksup[ikl - 1]; ++i) ntimes[i - 1] = ntimes[i - 1] + 1;
        }
      }
      for (int i = 0; i < nk; ++i) {
        if (ntimes[i] > 0) {
          s1[i] = s1[i] / static_cast<float>(ntimes[i]);
          s2[i] = s2[i] / static_cast<float>(ntimes[i]);
        } else {
          s1[i] = s2[i] = zero;
        }
      }
      for (int ik = 1; ik <= nk; ++ik) s1[ik - 1] = s1[ik - 1] / f.sig[ik];
    }
    cta.sync();
    PFOR(ik0, nk) {
      const int ik = ik0 + 1;
      float v = zero;
      for (int is = (ik - 1) * nth + 1; is <= ik * nth; ++is) v = v + a[is - 1];
      const float asum = v * dth;
      if (asum > 1.E-8f) {
        for (int is = 1 + (ik - 1) * nth; is <= ik * nth; ++is) ddiag[is - 1] = s1[ik - 1] / asum;
        for (int is = 1 + (ik - 1) * nth; is <= ik * nth; ++is) pb2[is - 1] = s2[ik - 1] / asum;
      } else {
        for (int is = 1 + (ik - 1) * nth; is <= ik * nth; ++is) ddiag[is - 1] = pb2[is - 1] = zero;
      }
      bth0[ik - 1] = pb2[(ik - 1) * nth] > 0.001f ? 2.0f * p.ssdsbr : zero;
    }
    cta.sync();
    PFOR(i, nspec) {
      pb[i] = ((one - ssdsc[0]) * pb2[i]) * a[i] + ssdsc[0] * pb[i];
      brlambda[i] = pb[i] / kTwoPiSq;
      srhs[i] = ddiag[i] * a[i];
    }
    cta.sync();
  } else if (sdscase == 3) {
    // 2.c Romero 2019 (:2481-2520). BTH(1:NTH) is the scratch of one IK in the reference; here
    // each IK has its own row of bth, so the IK loop runs in parallel over IK.
    const float dth = p.dth;
    const float t28 = 28.0f / ssdsc[15];
    const float ko = (kGrav / (ustar * ustar)) / (t28 * t28);
    PFOR(ik0, nk) {
      const int ik = ik0 + 1;
      const int is0 = (ik - 1) * nth;
      const float kx = kk[ik - 1];
      const float kloc = dm::powf(kx, 2.0f - ssdsc[19]);
      const float k3 = (kx * kx) * kx;
      float* const bthk = bth + is0;
      for (int ith = 1; ith <= nth; ++ith)
        bthk[ith - 1] = max_r((a[is0 + ith - 1] * f.sig[ik]) * k3, .00000000000001f);
      float dirforcum = dlwmean;
      if (ssdsc[10] > zero) dirforcum = MSS(ik, 2);
      const float c = f.sig[ik] / kx;
      float sb = zero;
      for (int ith = 1; ith <= nth; ++ith) sb = sb + bthk[ith - 1] * dth;
      bth0[ik - 1] = sb;
      float* const lmod = pb + is0;  // LMODULATION of this IK
      if (ssdsc[17] > zero) {
        float cd, sd;
        dm::sincosf(dirforcum, &sd, &cd);
        const float pm = dm::powf(MSS(ik, 1) * kloc, ssdsc[13]);
        for (int ith = 1; ith <= nth; ++ith) {
          const float q = f.ecos[ith - 1] * cd + f.esin[ith - 1] * sd;
          lmod[ith - 1] = one + ssdsc[17] * (pm * (q * q));
        }
        for (int ith = 0; ith < nth; ++ith) lmod[ith] = dm::powf(lmod[ith], ssdsc[18]);
      } else {
        for (int ith = 0; ith < nth; ++ith) lmod[ith] = one;
      }
      const float fk = one + ssdsc[12] * dm::powf(max_r(kx / ko, one), ssdsc[14]);
      const float c9 = ssdsc[8], c13p1 = ssdsc[12] + one;
      for (int ith = 0; ith < nth; ++ith)
        brlambda[is0 + ith] =
            (((c9 * dm::expf(-(p.ssdsbr / bthk[ith]))) * fk) / c13p1) * lmod[ith];
      const float btover = sqrt_f(bth0[ik - 1]) - sqrt_f(p.ssdsbt);
      brm12[ik - 1] = ssdsc[1] * dm::powf(zero > btover ? zero : btover, 2.5f);
      for (int ith = 1; ith <= nth; ++ith) {
        const float x = copysignf(brlambda[is0 + ith - 1], btover);
        brlambda[is0 + ith - 1] = x > zero ? x : zero;
      }
      const float c2 = c * c;
      const float c5 = (c * c2) * c2;
      for (int ith = 1; ith <= nth; ++ith)
        srhs[is0 + ith - 1] =
            (((brm12[ik - 1] / kGrav2) * brlambda[is0 + ith - 1]) * c5) / f.sig[ik];
      for (int ith = 1; ith <= nth; ++ith)
        ddiag[is0 + ith - 1] = ((srhs[is0 + ith - 1] * p.ssdsbr) / max_r(bthk[ith - 1], 1.e-20f)) /
                               max_r(a[is0 + ith - 1], 1e-20f);
    }
    cta.sync();
  }

  // Wave-turbulence interaction and cumulative effect (:2533-2575).
  if ((ssdsc[2] != zero) || (ssdsc[4] != zero) || (ssdsc[20] != zero)) {
    const int dikcumul = sh.dikcumul;
    float cu, su;
    dm::sincosf(usdir, &su, &cu);
    PFOR(i, nspec) {
      const int ik = i / nth + 1, ith = i - (ik - 1) * nth + 1;
      if (ik >= ik1) {
        const int is = i + 1;
        float renewalfreq = zero;
        const float facturb2 = -(((f.sig[ik] * 2.0f) * kk[ik - 1]) * sh.facturb);
        const float dvisc = -(((ssdsc[20] * 4.0f) * kk[ik - 1]) * kk[ik - 1]);
        const float c = f.sig[ik] / kk[ik - 1];
        if (ssdsc[2] > zero && ik > dikcumul) {
          for (int ik2 = ik1; ik2 <= ik - dikcumul; ++ik2) {
            const float cc2 = f.sig[ik2] / kk[ik2 - 1];
            const int is2 = (ik2 - 1) * nth;
            const float cumulwiso = ((fabs_f(cc2 - c) * f.dsip[ik2]) / (cc2 * 0.5f)) * p.dth;
            float v = zero;
            for (int j = is2; j < is2 + nth; ++j) v = v + brlambda[j];
            renewalfreq = renewalfreq - cumulwiso * v;
          }
        }
        if (ssdsc[2] < zero && ik > dikcumul) {
          renewalfreq = zero;
          for (int ik2 = ik1; ik2 <= ik - dikcumul; ++ik2) {
            if (bth0[ik2 - 1] > p.ssdsbr) {
              const int is2 = (ik2 - 1) * nth;
              float v = zero;
              // CUMULW(IS2+J, IS) for the threads' consecutive IS are consecutive in the
              // transposed copy: one coalesced row per J, streamed past L1.
              const float* const row =
                  f.cumulw + static_cast<size_t>(is2) * f.cumulw_ld + (is - 1);
              for (int j = 1; j <= nth; ++j)
                v = v + ld_stream(row + static_cast<size_t>(j - 1) * f.cumulw_ld) *
                            brlambda[is2 + j - 1];
              renewalfreq = renewalfreq + v;
            }
          }
        }
        const float coswind = f.ecos[ith - 1] * cu + f.esin[ith - 1] * su;
        const float dturb = facturb2 * max_r(coswind, zero);
        const float diag2 = (ssdsc[2] * renewalfreq + dturb) + dvisc;
        ddiag[is - 1] = ddiag[is - 1] + diag2;
        srhs[is - 1] = srhs[is - 1] + a[is - 1] * diag2;
      }
    }
    cta.sync();
  }

  // Whitecap parameters (:2581-2650); an early return leaves WHITECAP as it came. COEF4, COEF5
  // and the mean foam thickness of each IK are independent over IK (parallel); the sums over IK
  // (the coverage recurrence, the air entrainment and the foam sum) stay serial in IK order.
  if (flogrd57 || flogrd58) {
    const int fl = ffloor(p.aaircmin);
    const int ikc = fl < nk ? fl : nk;
    float* const mftk = s1;  // S1 is free after the breaking cases: MFT of each IK
    PFOR(ik0, nk) {
      const int ik = ik0 + 1;
      if (ik <= ikc) {
        const float c = f.sig[ik] / kk[ik - 1];
        const int is0 = (ik - 1) * nth;
        float v = zero;
        for (int i = is0; i < is0 + nth; ++i) v = v + brlambda[i];
        coef4[ik - 1] = ((((((c * c) * v) * 2.0f) * kPi) / kGrav) * ssdsc[6]) * f.dden[ik - 1] /
                        (f.sig[ik] * cg[ik - 1]);
        const float pw = dm::powf(brm12[ik - 1] / ssdsc[1], 3.0f / 5.0f);
        float w = zero;
        for (int i = is0; i < is0 + nth; ++i) w = w + (brlambda[i] * (-ssdsc[1])) * pw;
        coef5[ik - 1] = ((((c * c) * c) * w) * p.aairgb / kGrav) * f.dden[ik - 1] /
                        (f.sig[ik] * cg[ik - 1]);
      } else {
        coef4[ik - 1] = zero;
        coef5[ik - 1] = zero;
      }
      if (flogrd58 && ik >= ik1) {
        const float tstr = kTstrFac / f.sig[ik];
        const float tmax = kTmaxFac / f.sig[ik];
        const float dt = tmax / 50.0f;
        float mft = zero;
        for (int it = 1; it <= 50; ++it) {
          const float t = static_cast<float>(it) * dt;
          if (t < tstr) {
            mft = mft + ((0.4f / (kk[ik - 1] * tstr)) * t) * dt;
          } else {
            mft = mft + ((0.4f / kk[ik - 1]) * dm::expf(-((t - tstr) / 3.8f))) * dt;
          }
        }
        mftk[ik - 1] = mft / tmax;
      }
    }
    cta.sync();
    if (cta.role(0)) {
      float wc0 = zero, wc1 = zero, wc3 = zero;
      if (flogrd57) {
        for (int ik = ik1; ik <= ikc; ++ik) {
          wc0 = wc0 + coef4[ik - 1] * (one - wc0);
          wc3 = wc3 + coef5[ik - 1];
        }
      }
      if (flogrd58) {
        for (int ik = ik1; ik <= nk; ++ik) wc1 = wc1 + coef4[ik - 1] * mftk[ik - 1];
      }
      whitecap[0] = wc0;
      whitecap[1] = wc1;
      whitecap[2] = zero;
      whitecap[3] = wc3;
    }
    cta.sync();
  }
}

}  // namespace pt
}  // namespace wwb
