// ww3-gpu_b200/csrc/st4_tables_kernel.cu
// INSIN4 on sm_100a (see st4_tables_kernel.cuh). Every table entry the reference computes in a
// loop iteration that writes only that entry becomes one thread; the loops that carry a value
// (the DCKI/QBI sums over KH, TAUHFT's and TAUHFT2's sums over J, TAUHFT2's friction velocity
// carried over every (ILEVTAIL, J), IKTAB's TOTO carried over IKL) stay serial inside their
// thread, in the reference's order. The arithmetic keeps the reference's operand order, one
// rounding per operation (the build has no fused multiply-add), and calls the device libm with
// the host glibc's bits (libm_dev.cuh) where the reference calls expf, logf, powf, cosf, tanhf.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/st4_insin4.cpp:96-264 (INSIN4), st4_tabu_stress.cpp:20-73
// (TABU_STRESS), st4_tabu_tauhf.cpp:18-76 (TABU_TAUHF), st4_tabu_tauhf2.cpp:25-101
// (TABU_TAUHF2); WW3 w3src4md.F90:1014-1831.
#include "st4_tables_kernel.cuh"

#include <cmath>

#include "libm_dev.cuh"
#include "wavnu2_dev.cuh"
#include "wwb_common.hpp"

namespace wwb {
namespace {

using st4::kIalpha;
using st4::kIlevTail;
using st4::kItauMax;
using st4::kIustar;
using st4::kJuMax;
using st4::kNdtab;
using st4::kNkd;
using st4::kNkhs;

// CONSTANTS and W3SRC4MD PARAMETERs (constants.F90:62-76, w3src4md.F90:61-71), each operation
// rounded to REAL as the Fortran's PARAMETER folding does.
constexpr float kGrav = 9.806f;
constexpr float kKappa = 0.40f;
constexpr float kPi = static_cast<float>(3.141592653589793);
constexpr float kRade = 180.0f / kPi;
constexpr float kUmax = 50.0f;
constexpr float kTauwMax = 2.2361f;
constexpr int kNkhi = 100;
constexpr int kFacKd2 = 1000;
constexpr float kFacKd1 = 1.01f;
constexpr float kKhsMax = 2.0f;
constexpr float kKhMax = 2.0f;
constexpr int kJtot = 250;  // TABU_TAUHF / TABU_TAUHF2 JTOT

// XT = TANH(FAC_KD1**(1-FAC_KD2)) at IKD = 1: gfortran evaluates this one at compile time with
// the exact power (the runtime chain of squarings differs by about 6e-6 relative). Here:
// tanh(1.01f**-999) computed exactly and rounded to float, 0x1.943dfep-15.
constexpr float kXtIkd1 = 0x1.943dfep-15f;

__device__ __forceinline__ float max_r(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float min_r(float a, float b) { return a < b ? a : b; }
// std::max / std::min of the reference's host code: (a < b) ? b : a and (b < a) ? b : a.
__device__ __forceinline__ float std_max(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float std_min(float a, float b) { return (b < a) ? b : a; }

__device__ __forceinline__ float dexpf(float x) { return dm::expf_t<WWB_EXPF_FUSE>(x); }
__device__ __forceinline__ float dlogf(float x) { return dm::logf_t<WWB_LOGF_FUSE>(x); }

/// x**n for an INTEGER n at run time as gfortran -O3 computes it (libgcc's power by repeated
/// squaring, one float rounding per step, 1/y for a negative n).
__device__ __forceinline__ float powi(float x, int n) {
  unsigned m = n < 0 ? static_cast<unsigned>(-n) : static_cast<unsigned>(n);
  float y = (m & 1u) ? x : 1.0f;
  while ((m >>= 1u) != 0u) {
    x = x * x;
    if (m & 1u) y = y * x;
  }
  return n < 0 ? 1.0f / y : y;
}

// ------------------------------------------------------------------------------ TABU_STRESS
/// TAUT(I,J) = SQRT(TAU) after NITER = 10 Newton steps on the log profile with the
/// wave-supported stress (st4_tabu_stress.cpp:36-66); TAUT(I,0) = 0.
__global__ void taut_kernel(float aalpha, float zz0max, float zzwnd, float delu, float deltauw,
                            float* __restrict__ taut) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  constexpr int ni = kItauMax + 1, nj = kJuMax + 1;
  if (n >= ni * nj) return;
  const int i = n % ni, j = n / ni;
  if (j == 0) {
    taut[n] = 0.0f;
    return;
  }
  constexpr float kXm = 0.50f, kEps1 = 0.00001f, one = 1.0f;
  const float zt = static_cast<float>(i) * deltauw;
  const float ztauw = zt * zt;
  const float utop = static_cast<float>(j) * delu;
  const float wcd = sqrtf(0.0012875f);
  const float ustold = utop * wcd;
  float tauold = std_max(ustold * ustold, ztauw + kEps1);
  for (int iter = 1; iter <= 10; ++iter) {
    const float x = ztauw / tauold;
    float ust = sqrtf(tauold);
    float zz00 = aalpha * tauold / kGrav;
    if (zz0max != 0.0f) zz00 = std_min(zz00, zz0max);
    const float zz0 = zz00 / dm::powf(one - x, kXm);
    const float lg = dlogf(zzwnd / zz0);
    const float f = ust - kKappa * utop / lg;
    const float delf =
        one - kKappa * utop / (lg * lg) * 2.0f / ust * (one - 1.5f * x) / (one - x);
    ust = ust - f / delf;
    tauold = std_max(ust * ust, ztauw + kEps1);
  }
  taut[n] = sqrtf(tauold);
}

// ------------------------------------------------------------------------------ TABU_TAUHF
__device__ __forceinline__ float tauhf_weight(int j) {
  return (j == 1 || j == kJtot) ? 0.5f : 1.0f;
}

/// TAUHFT(K,L): the high-frequency stress integrated over J = 1..JTOT (st4_tabu_tauhf.cpp:48-70).
/// Thread = (K, L), K fastest (the table's column-major order).
__global__ void tauhf_kernel(float aalpha, float zz0max, float zzalp, float const1,
                             float omegac, float delust, float delalp,
                             float* __restrict__ tauhft) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  constexpr int nk = kIustar + 1;
  if (n >= nk * (kIalpha + 1)) return;
  const int k = n % nk, l = n / nk;
  const float x0 = 0.05f;
  const float ust = max_r(static_cast<float>(k) * delust, 0.000001f);
  float zz00 = ust * ust * aalpha / kGrav;
  if (zz0max != 0.0f) zz00 = min_r(zz00, zz0max);
  const float zz0 = zz00 * (1.0f + static_cast<float>(l) * delalp / aalpha);
  const float omegacc = max_r(omegac, x0 * kGrav / ust);
  const float yc = omegacc * sqrtf(zz0 / kGrav);
  const float dely = max_r((1.0f - yc) / static_cast<float>(kJtot), 0.0f);
  float t = 0.0f;
  for (int j = 1; j <= kJtot; ++j) {
    const float y = yc + static_cast<float>(j - 1) * dely;
    const float omega = y * sqrtf(kGrav / zz0);
    const float cm = kGrav / omega;
    const float zx = ust / cm + zzalp;
    const float zarg = min_r(kKappa / zx, 20.0f);
    const float zmu = min_r(kGrav * zz0 / (cm * cm) * dexpf(zarg), 1.0f);
    const float zlog = min_r(dlogf(zmu), 0.0f);
    const float zlog2 = zlog * zlog;
    const float zbeta = const1 * zmu * (zlog2 * zlog2);
    t = t + tauhf_weight(j) * zbeta / y * dely;
  }
  tauhft[n] = t;
}

// ------------------------------------------------------------------------------ TABU_TAUHF2
/// TAUHFT(K,L) and TAUHFT2(K,L,0:ILEVTAIL) (st4_tabu_tauhf2.cpp:50-98). TAUHFT is reset and
/// summed again for every ILEVTAIL from UST0 alone, so the value left is the one sum computed
/// here once. TAUHFT2's friction velocity UST is carried from one ILEVTAIL to the next (it is set
/// to UST0 only before the first), so each (K, L) is one serial chain of (ILEVTAIL+1)*JTOT steps.
__global__ void __launch_bounds__(128) tauhf2_kernel(float aalpha, float zzalp, float const1,
                                                     float omegac, float delust, float delalp,
                                                     float deltail, float* __restrict__ tauhft,
                                                     float* __restrict__ tauhft2) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  constexpr int nk = kIustar + 1, nl = kIalpha + 1;
  if (n >= nk * nl) return;
  const int k = n % nk, l = n / nk;
  const float g = kGrav, x0 = 0.05f;
  const float ust0 = max_r(static_cast<float>(k) * delust, 0.000001f);
  float ust = ust0;
  const float zz0 = ((aalpha + static_cast<float>(l) * delalp) * (ust0 * ust0)) / g;
  const float omegacc = max_r((x0 * g) / ust, omegac);
  const float yc = sqrtf(zz0 / g) * omegacc;
  const float dely = max_r((1.0f - yc) / static_cast<float>(kJtot), 0.0f);
  const float sgz = sqrtf(g / zz0);
  float t1 = 0.0f;
  for (int j = 1; j <= kJtot; ++j) {
    const float y = static_cast<float>(j - 1) * dely + yc;
    const float cm = g / (sgz * y);
    const float zx = ust0 / cm + zzalp;
    const float zarg = min_r(kKappa / zx, 20.0f);
    const float zmu = min_r(((zz0 * g) / (cm * cm)) * dexpf(zarg), 1.0f);
    const float zlog = min_r(dlogf(zmu), 0.0f);
    const float zl2 = zlog * zlog;
    const float zbeta = (const1 * zmu) * (zl2 * zl2);
    t1 = t1 + ((tauhf_weight(j) * zbeta) / y) * dely;
  }
  tauhft[n] = t1;
  const float tauw0 = ust0 * ust0;
  for (int i = 0; i <= kIlevTail; ++i) {
    const float levtail = static_cast<float>(i) * deltail;
    float t2 = 0.0f;
    float tauw = tauw0;
    for (int j = 1; j <= kJtot; ++j) {
      const float w = tauhf_weight(j);
      const float y = static_cast<float>(j - 1) * dely + yc;
      const float cm = g / (sgz * y);
      const float zx = ust / cm + zzalp;
      const float zarg = min_r(kKappa / zx, 20.0f);
      const float zmu = min_r(((zz0 * g) / (cm * cm)) * dexpf(zarg), 1.0f);
      const float zlog = min_r(dlogf(zmu), 0.0f);
      const float zl2 = zlog * zlog;
      const float zbeta = (const1 * zmu) * (zl2 * zl2);
      const float r = ust / ust0;
      t2 = t2 + (((w * zbeta) * (r * r)) / y) * dely;
      tauw = tauw - ((((w * (ust * ust)) * zbeta) * levtail) / y) * dely;
      ust = sqrtf(max_r(tauw, 0.0f));
    }
    tauhft2[n + static_cast<size_t>(i) * nk * nl] = t2;
  }
}

// ----------------------------------------------------------------- SATINDICES, SATWEIGHTS
/// SATINDICES(ROW, ITH) and SATWEIGHTS(ROW, ITH) (st4_insin4.cpp:113-144): for ITH <= NTH and
/// ROW <= 2*SDSNTH+1 the direction I = ITH-SDSNTH+ROW-1 wrapped into 1..NTH and
/// COS(TH(ITH)-TH(J))**SSDSCOS; the other entries keep 1 and 0 (1 and 1 when SSDSDTH >= 180).
__global__ void sat_kernel(int nsat, int mth, int nth, int sdsnth, int sat, float ssdscos,
                           const float* __restrict__ th, float* __restrict__ satweights,
                           int* __restrict__ satindices) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nsat * mth) return;
  const int row = n % nsat + 1, ith = n / nsat + 1;
  int idx = 1;
  float wt = sat ? 0.0f : 1.0f;
  if (sat && ith <= nth && row <= 2 * sdsnth + 1) {
    const int i_int = ith - sdsnth + row - 1;
    int j_int = i_int;
    if (i_int < 1) j_int = i_int + nth;
    if (i_int > nth) j_int = i_int - nth;
    idx = j_int;
    float sn, cs;
    dm::sincosf(th[ith - 1] - th[j_int - 1], &sn, &cs);
    wt = dm::powf(cs, ssdscos);
  }
  satindices[n] = idx;
  satweights[n] = wt;
}

// ----------------------------------------------------------------------------------- IKTAB
/// IKTAB(IKL, ID) for one depth ID = 1..NDTAB (st4_insin4.cpp:152-190): the index of SIG nearest
/// to the frequency of the wavenumber (BSUP/BINF)**2 K(SIG(IKL), ID), with the reference's
/// TOTO carried over IKL. Rows past NK stay 0 (the array is zeroed first).
__global__ void iktab_kernel(int nk, int mk, float binf, float bsup,
                             const float* __restrict__ sig, int* __restrict__ iktab) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (id > kNdtab) return;
  int toto = 0;
  const float prof = static_cast<float>(id);
  int* col = iktab + static_cast<size_t>(id - 1) * mk;
  for (int ikl = 1; ikl <= nk; ++ikl) {
    float kik = 0.0f, cgg = 0.0f;
    disp::wavnu2(sig[ikl], prof, kik, cgg, 1e-7f, 15);
    const float k1 = kik;
    const float r = bsup / binf;
    const float k2 = (r * r) * k1;
    const float sigtab = sqrtf(kGrav * k2 * dm::tanhf(k2 * static_cast<float>(id)));
    int v = col[ikl - 1];
    if (sigtab <= sig[1]) v = 1;
    if (sigtab > sig[nk]) {
      v = nk + toto;
      toto = 1;
    }
    for (int ik = 1; ik <= nk - 1; ++ik) {
      if (sig[ik] < sigtab && sig[ik + 1] >= sigtab) {
        const float diff1 = sigtab - sig[ik];
        const float diff2 = sig[ik + 1] - sigtab;
        v = (diff1 < diff2) ? ik : ik + 1;
      }
    }
    col[ikl - 1] = v;
  }
}

// ------------------------------------------------------------------------------- DCKI, QBI
/// DCKI(IKHS, IKD) and QBI(IKHS, IKD) for one IKD per block (st4_insin4.cpp:193-236). The sums
/// over IKH run in the reference's order per thread; the factors that depend on (IKH, IKD) only
/// (1 - EXP(-(KH/(GAM*XT))**SSDSPBK) and EPS) are the same bits for every IKHS and are computed
/// once per block, as are the running sums KHS (over IKHS) and KH (over IKH), which the
/// reference accumulates in REAL.
__global__ void __launch_bounds__(256) dcki_kernel(float ssdsabk, float ssdspbk, float ssdsbck,
                                                   float ssdshck, float* __restrict__ dcki,
                                                   float* __restrict__ qbi) {
  __shared__ float khs_s[kNkhs];
  __shared__ float kh_s[kNkhi], wf_s[kNkhi], ep_s[kNkhi];
  const int ikd = blockIdx.x + 1;
  const float dhs = kKhsMax / static_cast<float>(kNkhs);
  const float dkh = kKhMax / static_cast<float>(kNkhi);
  float xt, sqgxt;
  if (ikd == 1) {
    xt = kXtIkd1;
  } else {
    xt = dm::tanhf(powi(kFacKd1, ikd - kFacKd2));
  }
  sqgxt = sqrtf(kGrav / xt);
  const float xt2 = xt * xt;
  const float xt3 = xt2 * xt;
  float gam = 1.0314f * xt3 - 1.9958f * xt2 + 1.5522f * xt + 0.1885f;
  gam = gam / 2.15f;
  if (threadIdx.x == 0) {
    float khs = 0.0f;
    for (int i = 0; i < kNkhs; ++i) {
      khs = khs + dhs;
      khs_s[i] = khs;
    }
  } else if (threadIdx.x == 32) {
    float kh = 0.0f;
    for (int i = 0; i < kNkhi; ++i) {
      kh = kh + dkh;
      kh_s[i] = kh;
    }
  }
  __syncthreads();
  if (threadIdx.x < kNkhi) {
    const float kh = kh_s[threadIdx.x];
    wf_s[threadIdx.x] = 1.0f - dexpf(-(dm::powf(kh / (gam * xt), ssdspbk)));
    ep_s[threadIdx.x] =
        -((dm::powf((ssdsbck / dm::powf(xt, ssdshck)) * kh, 3.0f)) / 4.0f) * sqgxt;
  }
  __syncthreads();
  const float sqrt2 = sqrtf(2.0f);
  for (int i = threadIdx.x; i < kNkhs; i += blockDim.x) {
    const float khs = khs_s[i];
    const float s = khs / (sqrt2 * gam * xt);
    const float ss = ssdsabk * (s * s);
    float d = 0.0f, q = 0.0f;
#pragma unroll 4
    for (int ikh = 0; ikh < kNkhi; ++ikh) {
      const float kh = kh_s[ikh];
      const float qq = kh / khs;
      const float pr = (4.0f * kh / (khs * khs)) * dexpf(-(2.0f * (qq * qq)));
      const float w = ss * wf_s[ikh];
      d = d + pr * w * ep_s[ikh] * dkh;
      q = q + pr * w * dkh;
    }
    const size_t o = static_cast<size_t>(ikd - 1) * kNkhs + i;
    dcki[o] = d;
    qbi[o] = q > 1.0f ? 1.0f : q;
  }
}

// ---------------------------------------------------------------------------------- CUMULW
/// CUMULW(IS2, IS) (st4_insin4.cpp:243-263): for IK2 <= IK - DIKCUMUL the cumulative-breaking
/// weight SQRT(C**2 + C2**2 - 2 C C2 ECOS(1+|ITH2-ITH|)) DSIP(IK2) / (C2/2) DTH with C = g/SIG;
/// 0 elsewhere. One thread per entry, IS2 fastest (the array's column-major order).
__global__ void cumulw_kernel(int nk, int nth, int mspec, int dikcumul, float dth,
                              const float* __restrict__ sig, const float* __restrict__ dsip,
                              const float* __restrict__ ecos, float* __restrict__ cumulw) {
  const int is2 = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int is = blockIdx.y + 1;
  if (is2 > mspec) return;
  float v = 0.0f;
  if (is <= nk * nth && is2 <= nk * nth) {
    const int ik = (is - 1) / nth + 1, ith = (is - 1) % nth + 1;
    const int ik2 = (is2 - 1) / nth + 1, ith2 = (is2 - 1) % nth + 1;
    if (ik2 <= ik - dikcumul) {
      const float c = kGrav / sig[ik];
      const float c2 = kGrav / sig[ik2];
      const int d = ith2 > ith ? ith2 - ith : ith - ith2;
      v = sqrtf(c * c + c2 * c2 - 2.0f * c * c2 * ecos[d]) * dsip[ik2] / (0.5f * c2) * dth;
    }
  }
  cumulw[static_cast<size_t>(is - 1) * mspec + (is2 - 1)] = v;
}

__global__ void fill_kernel(int* __restrict__ a, int n, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

int blocks_of(long long n, int per) { return static_cast<int>((n + per - 1) / per); }

/// Fortran NINT of a REAL: the nearest integer, halves away from zero.
int nint_host(float x) { return static_cast<int>(std::lround(x)); }

}  // namespace

St4TablesPlan st4_tables_plan(const st4::Params& p, bool fltabs) {
  St4TablesPlan q{};
  const bool tabs = p.sintailpar[0] > 0.5f;
  q.taut = tabs && fltabs;
  q.tauhf2 = tabs && fltabs && p.ttauwshelter > 0.0f;
  q.tauhf = tabs && fltabs && !q.tauhf2;  // TABU_TAUHF2 rebuilds all of TAUHFT after it
  q.delust = p.delust;
  q.delalp = p.delalp;
  q.deltauw = p.deltauw;
  q.delu = p.delu;
  q.deltail = p.deltail;
  if (q.taut) {
    q.delu = kUmax / static_cast<float>(kJuMax);
    q.deltauw = kTauwMax / static_cast<float>(kItauMax);
  }
  if (tabs && fltabs) {
    const float alpham = 20.0f * p.aalpha;
    q.delust = 5.0f / static_cast<float>(kIustar);
    q.delalp = alpham / static_cast<float>(kIalpha);
    if (q.tauhf2) q.deltail = alpham / static_cast<float>(kIlevTail);
  }
  q.nsat = 2 * (p.mth / 2 - 1) + 1;
  q.sat = p.ssdsdth < 180.0f;
  if (q.sat) {
    const int a = nint_host(p.ssdsdth / (p.dth * kRade));
    const int b = p.nth / 2 - 1;
    q.sdsnth = a < b ? a : b;
  }
  q.bck = p.ssdsbck > 0.0f;
  q.cumul = p.ssdsc[2] < 0.0f;
  if (q.cumul) q.dikcumul = nint_host(p.ssdsbrf1 / (p.xfr - 1.0f));
  return q;
}

void launch_st4_tables(const st4::Params& p, const St4TablesPlan& q, const St4TablesIn& in,
                       const St4TablesOut& out, cudaStream_t s, cudaStream_t s2) {
  const float const1 = p.bbeta / (kKappa * kKappa);  // KAPPA**2 folded to KAPPA*KAPPA
  cudaEvent_t fork = nullptr, join = nullptr;
  if (q.tauhf2 && out.tauhft && out.tauhft2) {
    // TAUHFT2's chains are the longest work: they start first, on their own stream.
    float sigmax = 0.0f;
    WWB_CHECK(cudaMemcpyAsync(&sigmax, in.sig + p.nk, sizeof(float), cudaMemcpyDeviceToHost, s));
    WWB_CHECK(cudaStreamSynchronize(s));
    WWB_CHECK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    WWB_CHECK(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    WWB_CHECK(cudaEventRecord(fork, s));
    WWB_CHECK(cudaStreamWaitEvent(s2, fork, 0));
    const int n = (kIustar + 1) * (kIalpha + 1);
    tauhf2_kernel<<<blocks_of(n, 128), 128, 0, s2>>>(p.aalpha, p.zzalp, const1, sigmax,
                                                     q.delust, q.delalp, q.deltail, out.tauhft,
                                                     out.tauhft2);
    WWB_CHECK(cudaGetLastError());
    WWB_CHECK(cudaEventRecord(join, s2));
  }
  if (q.taut && out.taut) {
    const int n = (kItauMax + 1) * (kJuMax + 1);
    taut_kernel<<<blocks_of(n, 256), 256, 0, s>>>(p.aalpha, p.zz0max, p.zzwnd, q.delu,
                                                   q.deltauw, out.taut);
  }
  if (q.tauhf && out.tauhft) {
    float sigmax = 0.0f;
    WWB_CHECK(cudaMemcpyAsync(&sigmax, in.sig + p.nk, sizeof(float), cudaMemcpyDeviceToHost, s));
    WWB_CHECK(cudaStreamSynchronize(s));
    const int n = (kIustar + 1) * (kIalpha + 1);
    tauhf_kernel<<<blocks_of(n, 128), 128, 0, s>>>(p.aalpha, p.zz0max, p.zzalp, const1, sigmax,
                                                   q.delust, q.delalp, out.tauhft);
  }
  if (out.satweights && out.satindices) {
    const int n = q.nsat * p.mth;
    sat_kernel<<<blocks_of(n, 256), 256, 0, s>>>(q.nsat, p.mth, p.nth, q.sdsnth, q.sat ? 1 : 0,
                                                 p.ssdscos, in.th, out.satweights,
                                                 out.satindices);
  }
  const size_t ntab = static_cast<size_t>(kNkhs) * kNkd;
  if (q.bck) {
    if (out.iktab) {
      WWB_CHECK(cudaMemsetAsync(out.iktab, 0, sizeof(int) * p.mk * kNdtab, s));
      iktab_kernel<<<blocks_of(kNdtab, 64), 64, 0, s>>>(p.nk, p.mk, 1.0f - p.ssdsbint,
                                                        1.0f + p.ssdsbint, in.sig, out.iktab);
    }
    if (out.dcki && out.qbi)
      dcki_kernel<<<kNkd, 256, 0, s>>>(p.ssdsabk, p.ssdspbk, p.ssdsbck, p.ssdshck, out.dcki,
                                       out.qbi);
  } else {
    if (out.iktab) {
      const int n = p.mk * kNdtab;
      fill_kernel<<<blocks_of(n, 256), 256, 0, s>>>(out.iktab, n, 1);
    }
    if (out.dcki) WWB_CHECK(cudaMemsetAsync(out.dcki, 0, sizeof(float) * ntab, s));
    if (out.qbi) WWB_CHECK(cudaMemsetAsync(out.qbi, 0, sizeof(float) * ntab, s));
  }
  if (out.cumulw) {
    const size_t nc = static_cast<size_t>(p.mspec) * p.mspec;
    if (q.cumul) {
      dim3 grid(blocks_of(p.mspec, 256), p.mspec);
      cumulw_kernel<<<grid, 256, 0, s>>>(p.nk, p.nth, p.mspec, q.dikcumul, p.dth, in.sig,
                                         in.dsip, in.ecos, out.cumulw);
    } else {
      WWB_CHECK(cudaMemsetAsync(out.cumulw, 0, sizeof(float) * nc, s));
    }
  }
  WWB_CHECK(cudaGetLastError());
  if (join) {
    WWB_CHECK(cudaStreamWaitEvent(s, join, 0));
    WWB_CHECK(cudaEventDestroy(fork));
    WWB_CHECK(cudaEventDestroy(join));
  }
}

}  // namespace wwb
