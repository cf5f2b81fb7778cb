// ww3-gpu_b200/csrc/mlp_ops.cu
// Element-wise kernels of the learned DIA surrogate (declared and explained in mlp_ops.cuh).
// None of this is bit-exact work: it is the approximate path, measured against the FP64 DIA at
// the end of this file, so fused multiply-adds and CUDA's own math functions are used freely.
#include <cuda_bf16.h>

#include <cmath>

#include "mlp.cuh"
#include "mlp_ops.cuh"
#include "wwb_common.hpp"

namespace wwb {
namespace mlp {
namespace {

constexpr double kPi = 3.141592653589793;
constexpr double kGrav = 9.806;  // the reference's GRAV (kokkos/src/ww_kokkos/st4_params.hpp:28)
constexpr float kTpiInvF = static_cast<float>(1.0 / (2.0 * 3.141592653589793));
constexpr float kInputFloor = 1e-6f;  // U + floor before the log
constexpr float kInputScale = 1.0f / 7.0f;
constexpr int kThreads = 256;

/// splitmix64's output function (S. Vigna, public domain): a counter-based generator, so every
/// point's draws depend only on (seed, point index, draw number).
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double uniform(uint64_t seed, uint64_t i, uint32_t j) {
  const uint64_t h = mix64(mix64(seed) ^ (i * 0x100000001B3ull + j * 0x9E3779B97F4A7C15ull));
  return static_cast<double>(h >> 11) * 0x1.0p-53;
}

template <class T>
__device__ __forceinline__ T block_sum(T v, T* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  T t = 0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : T(0);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) red[0] = t;
  }
  __syncthreads();
  t = red[0];
  __syncthreads();
  return t;
}

/// CONS of W3SNL1 section 1 (snl1_team.hpp:386-390) in float with CUDA's expf.
__device__ __forceinline__ float cons_of(const SurGrid& g, float kd) {
  const float x0 = g.kdcon * kd;
  const float x = x0 < g.kdmn ? g.kdmn : x0;
  const float y = g.snls3 * x;
  const float x2 = -1.e15f < y ? y : -1.e15f;
  return g.snlc1 * (1.0f + g.snls1 / x * (1.0f - g.snls2 * x) * expf(x2));
}

// ------------------------------------------------------------------------------ synthetic data

__device__ double jonswap(double f, double fp, double gam) {
  const double sg = f <= fp ? 0.07 : 0.09;
  const double r = exp(-(f - fp) * (f - fp) / (2.0 * sg * sg * fp * fp));
  const double q = fp / f;
  return pow(f, -5.0) * exp(-1.25 * q * q * q * q) * pow(gam, r);
}

__global__ void synth_kernel(SurGrid g, SynthDraw dr, long long p0, int npts, float* a,
                             float* cg, float* kdm) {
  const int ip = blockIdx.x;
  if (ip >= npts) return;
  __shared__ double ef1[64], ef2[64], cgk[64], kdk[64], dir1[64], dir2[64];
  __shared__ double tot[6];
  const int nk = g.nk, nth = g.nth, tid = threadIdx.x;
  const uint64_t gi = static_cast<uint64_t>(p0 + ip);
  const double hs = 0.5 + 7.5 * uniform(dr.seed, gi, 0);
  const double fp = 0.06 + 0.14 * uniform(dr.seed, gi, 1);
  const double gam = 1.0 + 4.0 * uniform(dr.seed, gi, 2);
  const double spr = 2.0 + 18.0 * uniform(dr.seed, gi, 3);
  const double thm = 2.0 * kPi * uniform(dr.seed, gi, 4);
  double dep = dr.dmin;
  if (dr.dmax > dr.dmin)
    dep = exp(log(dr.dmin) + (log(dr.dmax) - log(dr.dmin)) * uniform(dr.seed, gi, 5));
  const bool swell = uniform(dr.seed, gi, 6) < dr.bimodal;
  const double hs2 = 0.5 + 2.5 * uniform(dr.seed, gi, 7);
  const double fp2 = 0.05 + 0.04 * uniform(dr.seed, gi, 8);
  const double thm2 = 2.0 * kPi * uniform(dr.seed, gi, 9);
  for (int k = tid; k < nk; k += blockDim.x) {
    const double s = g.sig[k], f = s / (2.0 * kPi);
    ef1[k] = jonswap(f, fp, gam) / (2.0 * kPi);
    ef2[k] = swell ? jonswap(f, fp2, 3.3) / (2.0 * kPi) : 0.0;
    // k from s^2 = g k tanh(k d) by Newton from the deep-water value.
    double wk = s * s / kGrav;
    for (int it = 0; it < 30; ++it) {
      const double kd = fmin(wk * dep, 40.0);
      const double t = tanh(kd);
      const double f0 = kGrav * wk * t - s * s;
      const double f1 = kGrav * t + kGrav * wk * dep * (1.0 - t * t);
      wk -= f0 / f1;
    }
    const double kd = wk * dep;
    cgk[k] = 0.5 * s / wk * (1.0 + 2.0 * kd / sinh(fmin(2.0 * kd, 80.0)));
    kdk[k] = kd;
  }
  for (int t = tid; t < nth; t += blockDim.x) {
    const double th = t * static_cast<double>(g.dth);
    const double c1 = cos(0.5 * (th - thm)), c2 = cos(0.5 * (th - thm2));
    dir1[t] = pow(c1 * c1, spr);
    dir2[t] = pow(c2 * c2, 20.0);
  }
  __syncthreads();
  if (tid == 0) {
    const double xfr = g.xfr, dth = g.dth;
    double d1 = 0, d2 = 0, m1 = 0, m2 = 0;
    for (int t = 0; t < nth; ++t) {
      d1 += dir1[t];
      d2 += dir2[t];
    }
    for (int k = 0; k < nk; ++k) {
      const double dsii = 0.5 * static_cast<double>(g.sig[k]) * (xfr - 1.0 / xfr);
      m1 += ef1[k] * dsii;
      m2 += ef2[k] * dsii;
    }
    const double c1 = m1 > 0 ? (hs / 4.0) * (hs / 4.0) / m1 / (d1 * dth) : 0.0;
    const double c2 = (swell && m2 > 0) ? (hs2 / 4.0) * (hs2 / 4.0) / m2 / (d2 * dth) : 0.0;
    double esum = 0, ekd = 0;
    for (int k = 0; k < nk; ++k) {
      const double e = ef1[k] * c1 * d1 + ef2[k] * c2 * d2;
      esum += e;
      ekd += e * kdk[k];
    }
    tot[0] = c1;
    tot[1] = c2;
    tot[2] = esum > 0 ? ekd / esum : 0.0;
  }
  __syncthreads();
  const double c1 = tot[0], c2 = tot[1];
  const size_t nspec = static_cast<size_t>(nk) * nth;
  for (int i = tid; i < nk * nth; i += blockDim.x) {
    const int k = i / nth, t = i % nth;
    const double e = ef1[k] * dir1[t] * c1 + ef2[k] * dir2[t] * c2;
    a[ip * nspec + i] = static_cast<float>(e * cgk[k] / static_cast<double>(g.sig[k]));
  }
  for (int k = tid; k < nk; k += blockDim.x) cg[static_cast<size_t>(ip) * nk + k] = static_cast<float>(cgk[k]);
  if (tid == 0) kdm[ip] = static_cast<float>(tot[2]);
}

// ------------------------------------------------------------------------- input normalisation

/// ln of the quadrature weight DDEN(k) = DTH * DSII(k) * SIG(k), DSII = SIG (XFR - 1/XFR) / 2.
__device__ __forceinline__ float ln_dden(const SurGrid& g, float sig) {
  return logf(g.dth * 0.5f * sig * (g.xfr - 1.0f / g.xfr) * sig);
}

__device__ __forceinline__ float warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

constexpr int kPointsPerCta = 8;  // one warp per sea point in the pre- and post-processing

/// Floats of shared memory per warp of prep_kernel.
__host__ __device__ inline int prep_floats(int nspec, int nk, int nth) {
  return nspec + 4 * nk + nth;
}

__global__ void __launch_bounds__(32 * kPointsPerCta)
    prep_kernel(SurGrid g, int npts, const float* __restrict__ a, const float* __restrict__ cg,
                const float* __restrict__ kdm, __nv_bfloat16* __restrict__ x, int ldx,
                float* __restrict__ ps, int* __restrict__ shift, float* __restrict__ dzero,
                float* __restrict__ gzero) {
  extern __shared__ float sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ip = blockIdx.x * kPointsPerCta + warp;
  if (ip >= npts) return;  // warp-uniform: the rest of the kernel is per warp
  const int nk = g.nk, nth = g.nth, nspec = g.nspec;
  float* const ue = sm + static_cast<size_t>(warp) * prep_floats(nspec, nk, nth);
  float* const rcon = ue + nspec;  // nk: 1 / CONX
  float* const dsum = rcon + nk;   // nth: the spectrum summed over frequency per direction
  float* const rmax = dsum + nth;  // nk: largest UE of each row
  float* const lw = rmax + nk;     // nk: scratch per row
  float* const lam = lw + nk;      // nk
  const float* ap = a + static_cast<size_t>(ip) * nspec;
  const float* cgp = cg + static_cast<size_t>(ip) * nk;
  float* pp = ps + static_cast<size_t>(ip) * 2 * nk;
  for (int k = lane; k < nk; k += 32) rcon[k] = __ldg(g.sig + k) / (kTpiInvF * __ldg(cgp + k));
  __syncwarp();
  // UE = A / CONX, four bins per load (NTH a multiple of 4: the four share a row).
  float mx = 0.0f;
  if ((nth & 3) == 0 && (reinterpret_cast<uintptr_t>(ap) & 15) == 0) {
    const float4* a4 = reinterpret_cast<const float4*>(ap);
    float4* u4 = reinterpret_cast<float4*>(ue);
    // Row of float4 q = lane + 32 t, tracked without a division per step.
    const int q4 = nth >> 2, dk = 32 / q4, dr = 32 % q4;
    int kq = lane / q4, rq = lane % q4;
    for (int q = lane; q < nspec / 4; q += 32) {
      float4 v = __ldg(a4 + q);
      const float r = rcon[kq];
      rq += dr;
      kq += dk;
      if (rq >= q4) {
        rq -= q4;
        ++kq;
      }
      v.x *= r;
      v.y *= r;
      v.z *= r;
      v.w *= r;
      u4[q] = v;
      mx = fmaxf(mx, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
    }
  } else {
    for (int i = lane; i < nspec; i += 32) {
      const float v = __ldg(ap + i) * rcon[i / nth];
      ue[i] = v;
      mx = fmaxf(mx, v);
    }
  }
  const float umax = warp_max(mx);
  __syncwarp();
  for (int t = lane; t < nth; t += 32) {
    float s = 0.0f;
    for (int k = 0; k < nk; ++k) s += ue[k * nth + t];
    dsum[t] = s;
  }
  const float floor = fmaxf(umax * 1e-12f, 1e-30f);
  for (int k = lane; k < nk; k += 32) {
    float m = 0.0f;
    const float* row = ue + k * nth;
    for (int t = 0; t < nth; ++t) m = fmaxf(m, row[t]);
    rmax[k] = m;
    // the row's largest cubic term, ln(AF11 u^3)
    lw[k] = 3.0f * __logf(fmaxf(m, floor)) + 11.0f * __logf(__ldg(g.sig + k) * kTpiInvF);
  }
  __syncwarp();
  // Dominant direction (lowest index on ties), then which side of it is heavier.
  float bv = -1.0f;
  int bi = 0;
  for (int t = lane; t < nth; t += 32)
    if (dsum[t] > bv) {
      bv = dsum[t];
      bi = t;
    }
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > bv || (ov == bv && oi < bi)) {
      bv = ov;
      bi = oi;
    }
  }
  float up = 0.0f, lo = 0.0f;
  for (int j = 1 + lane; j < (nth + 1) / 2; j += 32) {
    int cu = bi + j, cl = bi - j;
    if (cu >= nth) cu -= nth;
    if (cl < 0) cl += nth;
    up += dsum[cu];
    lo += dsum[cl];
  }
  up = warp_sum(up);
  lo = warp_sum(lo);
  const int packed = bi | (lo > up ? 1 << 16 : 0);
  const float kd = __ldg(kdm + ip);
  const float cons = cons_of(g, kd);
  const float lcons = __logf(cons);
  // lambda(k) = ln CONS + ln CONX(k) + the largest cubic term within kReach rows of k (the rows
  // whose quadruplets reach row k): S(k, .) e^-lambda is of order one.
  constexpr int kReach = 5;
  for (int k = lane; k < nk; k += 32) {
    float l = -INFINITY;
    for (int q = max(0, k - kReach); q <= min(nk - 1, k + kReach); ++q) l = fmaxf(l, lw[q]);
    lam[k] = umax > 0.0f ? lcons - __logf(rcon[k]) + l : -1e30f;
  }
  __syncwarp();
  // The row's weight in the Hs tendency, e^lambda DDEN / CG, scaled by its largest value.
  float wmax = -INFINITY;
  for (int k = lane; k < nk; k += 32) {
    lw[k] = lam[k] + ln_dden(g, __ldg(g.sig + k)) - __logf(__ldg(cgp + k));
    wmax = fmaxf(wmax, lw[k]);
  }
  wmax = warp_max(wmax);
  for (int k = lane; k < nk; k += 32) {
    pp[k] = lam[k];
    pp[nk + k] = umax > 0.0f ? __expf(lw[k] - wmax) : 0.0f;
  }
  if (lane == 0) shift[ip] = packed;
  // The network input, row by row, two canonical columns per lane.
  const float inv = umax > 0.0f ? 1.0f / umax : 0.0f;
  __nv_bfloat16* xr = x + static_cast<size_t>(ip) * ldx;
  const int sh = packed & 0xFFFF;
  const bool flip = (packed >> 16) != 0;
  auto col = [&](int j) {
    int c = flip ? sh - j : sh + j;
    if (c >= nth) c -= nth;
    if (c < 0) c += nth;
    return c;
  };
  if ((nth & 1) == 0) {
    // Pairs of canonical bins (2p, 2p + 1), p = lane, lane + 32, ...: both in row k, column j.
    int j = (2 * lane) % nth, k = (2 * lane) / nth;
    const int dk = 64 / nth, dj = 64 % nth;
    for (int i = 2 * lane; i < nspec; i += 64) {
      const float* row = ue + k * nth;
      const float u0 = row[col(j)] * inv, u1 = row[col(j + 1)] * inv;
      const float x0 = __logf(u0 + kInputFloor) * kInputScale + 1.0f;
      const float x1 = __logf(u1 + kInputFloor) * kInputScale + 1.0f;
      *reinterpret_cast<__nv_bfloat162*>(xr + i) = __floats2bfloat162_rn(x0, x1);
      j += dj;
      k += dk;
      if (j >= nth) {
        j -= nth;
        ++k;
      }
    }
  } else {
    for (int k = 0; k < nk; ++k)
      for (int j = lane; j < nth; j += 32)
        xr[k * nth + j] =
            __float2bfloat16_rn(__logf(ue[k * nth + col(j)] * inv + kInputFloor) * kInputScale + 1.0f);
  }
  // Depth features: ln kdmean and the relative depth factor of CONS; zero padding.
  for (int i = nspec + lane; i < g.din; i += 32) {
    float v = 0.0f;
    if (i == nspec) v = __logf(fmaxf(kd, 1e-2f)) * 0.2f;
    if (i == nspec + 1) v = cons / g.snlc1 - 1.0f;
    xr[i] = __float2bfloat16_rn(v);
  }
  // The gated path's zeros: the point's D and its two gate sums.
  if (dzero)
    for (int i = lane; i < nspec; i += 32) dzero[static_cast<size_t>(ip) * nspec + i] = 0.0f;
  if (gzero && lane == 0) {
    gzero[2 * static_cast<size_t>(ip)] = 0.0f;
    gzero[2 * static_cast<size_t>(ip) + 1] = 0.0f;
  }
}


/// prep_kernel for one grid shape known at compile time (NK rows of NTH directions, 32 <= NK
/// <= 64, NTH a multiple of 4), with the same outputs. One warp per sea point; lane k owns
/// frequency row k (and row k + 32): it reads the row with 16-byte loads, scales it and keeps
/// its maximum in registers, and later writes the row's network inputs. The spectrum is kept in
/// shared memory with rows NTH + 1 floats apart, so lanes reading the same column of their rows
/// hit different banks. Column sums run one lane per direction, in row order as in prep_kernel.
template <int NK, int NTH>
__global__ void __launch_bounds__(32 * kPointsPerCta)
    prep_rows_kernel(SurGrid g, int npts, const float* __restrict__ a,
                     const float* __restrict__ cg, const float* __restrict__ kdm,
                     __nv_bfloat16* __restrict__ x, int ldx, float* __restrict__ ps,
                     int* __restrict__ shift, float* __restrict__ dzero,
                     float* __restrict__ gzero) {
  static_assert(NK >= 32 && NK <= 64 && NTH % 4 == 0, "prep_rows_kernel shape");
  constexpr int NSPEC = NK * NTH, LD = NTH + 1, Q = NTH / 4;
  __shared__ float sm_ue[kPointsPerCta][NK * LD];
  __shared__ float sm_lw[kPointsPerCta][NK];
  __shared__ float sm_ds[kPointsPerCta][NTH];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ip = blockIdx.x * kPointsPerCta + warp;
  if (ip >= npts) return;  // warp-uniform
  float* const ue = sm_ue[warp];
  float* const lw = sm_lw[warp];
  float* const ds = sm_ds[warp];
  const float* ap = a + static_cast<size_t>(ip) * NSPEC;
  const float* cgp = cg + static_cast<size_t>(ip) * NK;
  float* pp = ps + static_cast<size_t>(ip) * 2 * NK;

  // UE = A / CONX row by row (lane k: rows k and k + 32), each row's largest value.
  float rc[2] = {0.0f, 0.0f}, rmx[2] = {0.0f, 0.0f};
  float mx = 0.0f;
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int k = lane + 32 * r;
    if (k < NK) {
      const float rk = __ldg(g.sig + k) / (kTpiInvF * __ldg(cgp + k));
      rc[r] = rk;
      const float4* row = reinterpret_cast<const float4*>(ap + k * NTH);
      float* const u = ue + k * LD;
      float m = 0.0f;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        float4 v = __ldg(row + q);
        v.x *= rk;
        v.y *= rk;
        v.z *= rk;
        v.w *= rk;
        u[4 * q] = v.x;
        u[4 * q + 1] = v.y;
        u[4 * q + 2] = v.z;
        u[4 * q + 3] = v.w;
        m = fmaxf(m, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
      }
      rmx[r] = m;
      mx = fmaxf(mx, m);
    }
  }
  const float umax = warp_max(mx);
  const float floor = fmaxf(umax * 1e-12f, 1e-30f);
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int k = lane + 32 * r;
    if (k < NK)
      lw[k] = 3.0f * __logf(fmaxf(rmx[r], floor)) + 11.0f * __logf(__ldg(g.sig + k) * kTpiInvF);
  }
  __syncwarp();
  for (int t = lane; t < NTH; t += 32) {
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < NK; ++k) s += ue[k * LD + t];
    ds[t] = s;
  }
  __syncwarp();
  // Dominant direction (lowest index on ties), then which side of it is heavier.
  float bv = -1.0f;
  int bi = 0;
  for (int t = lane; t < NTH; t += 32)
    if (ds[t] > bv) {
      bv = ds[t];
      bi = t;
    }
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > bv || (ov == bv && oi < bi)) {
      bv = ov;
      bi = oi;
    }
  }
  float up = 0.0f, lo = 0.0f;
  for (int j = 1 + lane; j < (NTH + 1) / 2; j += 32) {
    int cu = bi + j, cl = bi - j;
    if (cu >= NTH) cu -= NTH;
    if (cl < 0) cl += NTH;
    up += ds[cu];
    lo += ds[cl];
  }
  up = warp_sum(up);
  lo = warp_sum(lo);
  const int packed = bi | (lo > up ? 1 << 16 : 0);
  const float kd = __ldg(kdm + ip);
  const float cons = cons_of(g, kd);
  const float lcons = __logf(cons);
  // lambda(k) and the Hs-tendency weights, as prep_kernel.
  constexpr int kReach = 5;
  float lam[2] = {0.0f, 0.0f}, wl[2] = {-INFINITY, -INFINITY};
  float wmax = -INFINITY;
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int k = lane + 32 * r;
    if (k < NK) {
      float l = -INFINITY;
      for (int q = max(0, k - kReach); q <= min(NK - 1, k + kReach); ++q) l = fmaxf(l, lw[q]);
      lam[r] = umax > 0.0f ? lcons - __logf(rc[r]) + l : -1e30f;
      wl[r] = lam[r] + ln_dden(g, __ldg(g.sig + k)) - __logf(__ldg(cgp + k));
      wmax = fmaxf(wmax, wl[r]);
    }
  }
  wmax = warp_max(wmax);
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int k = lane + 32 * r;
    if (k < NK) {
      pp[k] = lam[r];
      pp[NK + k] = umax > 0.0f ? __expf(wl[r] - wmax) : 0.0f;
    }
  }
  if (lane == 0) shift[ip] = packed;
  // The network input in canonical order: lane k writes row k (four bins per 8-byte store),
  // then the rows from 32 up are shared by all lanes.
  const float inv = umax > 0.0f ? 1.0f / umax : 0.0f;
  __nv_bfloat16* xr = x + static_cast<size_t>(ip) * ldx;
  const int sh = packed & 0xFFFF;
  const bool flip = (packed >> 16) != 0;
  auto xval = [&](float u) { return __logf(u * inv + kInputFloor) * kInputScale + 1.0f; };
  {
    const float* row = ue + lane * LD;
    const int step = flip ? -1 : 1;
    int c = sh;
#pragma unroll
    for (int j = 0; j < NTH; j += 4) {
      float v[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        v[e] = xval(row[c]);
        c += step;
        if (c >= NTH) c -= NTH;
        if (c < 0) c += NTH;
      }
      const __nv_bfloat162 b0 = __floats2bfloat162_rn(v[0], v[1]);
      const __nv_bfloat162 b1 = __floats2bfloat162_rn(v[2], v[3]);
      uint2 pk;
      pk.x = *reinterpret_cast<const unsigned*>(&b0);
      pk.y = *reinterpret_cast<const unsigned*>(&b1);
      *reinterpret_cast<uint2*>(xr + lane * NTH + j) = pk;
    }
  }
  for (int i = lane; i < (NK - 32) * NTH; i += 32) {
    const int k = 32 + i / NTH, j = i % NTH;
    int c = flip ? sh - j : sh + j;
    if (c >= NTH) c -= NTH;
    if (c < 0) c += NTH;
    xr[k * NTH + j] = __float2bfloat16_rn(xval(ue[k * LD + c]));
  }
  // Depth features: ln kdmean and the relative depth factor of CONS; zero padding.
  for (int i = NSPEC + lane; i < g.din; i += 32) {
    float v = 0.0f;
    if (i == NSPEC) v = __logf(fmaxf(kd, 1e-2f)) * 0.2f;
    if (i == NSPEC + 1) v = cons / g.snlc1 - 1.0f;
    xr[i] = __float2bfloat16_rn(v);
  }
  // The gated path's zeros: the point's D (16-byte stores) and its two gate sums.
  if (dzero) {
    float4* const d4 = reinterpret_cast<float4*>(dzero + static_cast<size_t>(ip) * NSPEC);
    for (int i = lane; i < NSPEC / 4; i += 32) d4[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  if (gzero && lane == 0) {
    gzero[2 * static_cast<size_t>(ip)] = 0.0f;
    gzero[2 * static_cast<size_t>(ip) + 1] = 0.0f;
  }
}

// ------------------------------------------------------------------------------ target side

__global__ void rowscale_kernel(SurGrid g, int npts, const float* __restrict__ s,
                                const float* __restrict__ ps, double* acc,
                                unsigned long long* cnt) {
  __shared__ double rs[64];
  const int ip = blockIdx.x, tid = threadIdx.x, nk = g.nk, nth = g.nth;
  const float* pp = ps + static_cast<size_t>(ip) * 2 * nk;
  if (!(pp[0] > -1e29f)) return;  // an empty spectrum
  for (int k = tid; k < nk; k += blockDim.x) rs[k] = 0.0;
  __syncthreads();
  const float* sp = s + static_cast<size_t>(ip) * g.nspec;
  for (int i = tid; i < g.nspec; i += blockDim.x) {
    const int k = i / nth;
    const double v = static_cast<double>(sp[i]) * exp(-static_cast<double>(pp[k]));
    atomicAdd(&rs[k], v * v);
  }
  __syncthreads();
  for (int k = tid; k < nk; k += blockDim.x) atomicAdd(acc + k, rs[k]);
  if (tid == 0) atomicAdd(cnt, 1ull);
}

__global__ void targets_kernel(SurGrid g, int npts, const float* __restrict__ s,
                               const float* __restrict__ ps, const int* __restrict__ shift,
                               float* __restrict__ t, int ldt) {
  const int ip = blockIdx.x, tid = threadIdx.x, nk = g.nk, nth = g.nth;
  const float* pp = ps + static_cast<size_t>(ip) * 2 * nk;
  const int sh = shift[ip];
  const float* sp = s + static_cast<size_t>(ip) * g.nspec;
  float* tp = t + static_cast<size_t>(ip) * ldt;
  for (int i = tid; i < g.nspec; i += blockDim.x) {
    const int k = i / nth, j = i % nth;
    const double den = exp(static_cast<double>(pp[k])) * __ldg(g.rowscale + k);
    tp[i] = den > 0.0 ? static_cast<float>(static_cast<double>(sp[k * nth + orig_col(sh, j, nth)]) / den)
                      : 0.0f;
  }
}

// ------------------------------------------------------------------------ inference output side

__global__ void gate_kernel(GateParams gate, int npts, const float* __restrict__ gsum,
                            const float* __restrict__ head, int* __restrict__ accepted,
                            float* __restrict__ gv, int* __restrict__ rej_list,
                            int* __restrict__ nrej, int* __restrict__ nrej_total, int base) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= npts) return;
  const float r = gsum[2 * ip], gs = gsum[2 * ip + 1];
  const float h = head ? head[ip] : -INFINITY;
  const float resid = gs > 0.0f ? fabsf(r) / gs : 0.0f;
  const bool ok = isfinite(r) && isfinite(gs) && isfinite(h) && resid <= gate.energy &&
                  h <= gate.log_err;
  if (accepted) accepted[ip] = ok ? 1 : 0;
  if (gv) {
    gv[2 * ip] = h;
    gv[2 * ip + 1] = resid;
  }
  if (!ok) {
    rej_list[atomicAdd(nrej, 1)] = base + ip;
    if (nrej_total) atomicAdd(nrej_total, 1);
  }
}

// ------------------------------------------------------------------------------ training side

__global__ void loss_kernel(SurGrid g, LossWeights lw, int m, int nvalid,
                            const float* __restrict__ out, int ldo, const float* __restrict__ t,
                            int ldt, const float* __restrict__ ps, __nv_bfloat16* __restrict__ grad,
                            int ldg, float* __restrict__ loss) {
  __shared__ float red[32];
  __shared__ float wgt[64], dband[64], tband[64];
  const int ip = blockIdx.x, tid = threadIdx.x, nk = g.nk;
  const float* op = out + static_cast<size_t>(ip) * ldo;
  const float* tp = t + static_cast<size_t>(ip) * ldt;
  // The band terms need rows of NTH bins: the surrogate's targets (nvalid == NSPEC).
  const bool energy = ps != nullptr && nvalid == g.nspec && nk <= 64;
  if (energy) {
    const float* pp = ps + static_cast<size_t>(ip) * 2 * nk;
    for (int k = tid; k < nk; k += blockDim.x) {
      wgt[k] = __ldg(g.rowscale + k) * pp[nk + k];
      dband[k] = 0.0f;
      tband[k] = 0.0f;
    }
    __syncthreads();
  }
  float se = 0.0f;
  for (int i = tid; i < nvalid; i += blockDim.x) {
    const float dv = op[i] - tp[i];
    se += dv * dv;
    if (energy) {
      const int k = i / g.nth;
      atomicAdd(&dband[k], wgt[k] * dv);
      atomicAdd(&tband[k], wgt[k] * tp[i]);
    }
  }
  se = block_sum(se, red);
  // Per frequency band k: the error of the band's Hs (energy) tendency d(k) and the tendency
  // t(k); the band error is sum |d| / sum |t|, the loss term sum d^2 / (sum |t|)^2.
  float den = 0.0f, num = 0.0f, sq = 0.0f;
  if (energy) {
    __syncthreads();
    for (int k = 0; k < nk; ++k) {
      den += fabsf(tband[k]);
      num += fabsf(dband[k]);
      sq += dband[k] * dband[k];
    }
  }
  const bool have_e = energy && den > 1e-30f;
  const float band_err = have_e ? num / den : 0.0f;
  const float inv_m = 1.0f / static_cast<float>(m);
  const float c_mse = 2.0f * inv_m / static_cast<float>(nvalid);
  const float c_e = have_e ? lw.mu * 2.0f / (den * den) * inv_m : 0.0f;
  const bool head = lw.head && g.dout > nvalid;
  const float target_h = logf(band_err + 1e-3f);
  __nv_bfloat16* gp = grad + static_cast<size_t>(ip) * ldg;
  const int width = g.dout;
  for (int i = tid; i < width; i += blockDim.x) {
    float v = 0.0f;
    if (i < nvalid) {
      v = c_mse * (op[i] - tp[i]);
      if (have_e) {
        const int k = i / g.nth;
        v += c_e * dband[k] * wgt[k];
      }
    } else if (head && i == nvalid) {
      v = lw.lambda * 2.0f * (op[i] - target_h) * inv_m;
    }
    gp[i] = __float2bfloat16_rn(v);
  }
  if (tid == 0) {
    atomicAdd(loss + 0, se * inv_m / static_cast<float>(nvalid));
    if (have_e) atomicAdd(loss + 1, lw.mu * sq / (den * den) * inv_m);
    if (head) {
      const float h = op[nvalid] - target_h;
      atomicAdd(loss + 2, lw.lambda * h * h * inv_m);
    }
  }
}

__global__ void gather_kernel(int m, long long n, uint64_t seed, long long offset,
                              const __nv_bfloat16* __restrict__ xs, int ldx,
                              const float* __restrict__ ts, int ldt, const float* __restrict__ pss,
                              int ldp, __nv_bfloat16* __restrict__ xb, float* __restrict__ tb,
                              float* __restrict__ psb) {
  const int r = blockIdx.x;
  if (r >= m) return;
  long long src = offset + r;
  if (seed != 0) src = static_cast<long long>(mix64(mix64(seed) ^ static_cast<uint64_t>(r)) % static_cast<uint64_t>(n));
  const uint4* xsrc = reinterpret_cast<const uint4*>(xs + src * ldx);
  uint4* xdst = reinterpret_cast<uint4*>(xb + static_cast<size_t>(r) * ldx);
  for (int i = threadIdx.x; i < ldx / 8; i += blockDim.x) xdst[i] = __ldg(xsrc + i);
  const float4* tsrc = reinterpret_cast<const float4*>(ts + src * ldt);
  float4* tdst = reinterpret_cast<float4*>(tb + static_cast<size_t>(r) * ldt);
  for (int i = threadIdx.x; i < ldt / 4; i += blockDim.x) tdst[i] = __ldg(tsrc + i);
  for (int i = threadIdx.x; i < ldp; i += blockDim.x) psb[static_cast<size_t>(r) * ldp + i] = pss[src * ldp + i];
}

__global__ void transpose_kernel(const __nv_bfloat16* __restrict__ src, int rows, int cols,
                                 int lds, __nv_bfloat16* __restrict__ dst, int ldd) {
  __shared__ __nv_bfloat16 tile[32][34];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int rr = threadIdx.y; rr < 32; rr += 8) {
    const int r = r0 + rr, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[rr][threadIdx.x] = src[static_cast<size_t>(r) * lds + c];
  }
  __syncthreads();
  for (int cc = threadIdx.y; cc < 32; cc += 8) {
    const int c = c0 + cc, r = r0 + threadIdx.x;
    if (c < cols && r < rows) dst[static_cast<size_t>(c) * ldd + r] = tile[threadIdx.x][cc];
  }
}

__global__ void colsum_kernel(const __nv_bfloat16* __restrict__ gt, int n, int m, int ldt,
                              float* __restrict__ db) {
  const int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
  if (row >= n) return;
  const __nv_bfloat16* p = gt + static_cast<size_t>(row) * ldt;
  float acc = 0.0f;
  for (int i = lane * 8; i < m; i += 256) {
    const uint4 u = *reinterpret_cast<const uint4*>(p + i);
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w[q]));
      acc += f.x + f.y;
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) db[row] = acc;
}

__global__ void adamw_kernel(Adam h, int n, int k, float* __restrict__ w, float* __restrict__ m,
                             float* __restrict__ v, float* __restrict__ g,
                             __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wt,
                             int update) {
  __shared__ __nv_bfloat16 tile[32][34];
  const int c = blockIdx.x * 32 + threadIdx.x;
  for (int rr = threadIdx.y; rr < 32; rr += 8) {
    const int r = blockIdx.y * 32 + rr;
    if (r < n && c < k) {
      const size_t i = static_cast<size_t>(r) * k + c;
      float wi = w[i];
      if (update) {
        const float gi = g[i];
        const float mi = h.beta1 * m[i] + (1.0f - h.beta1) * gi;
        const float vi = h.beta2 * v[i] + (1.0f - h.beta2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        g[i] = 0.0f;
        wi = wi - h.lr * ((mi / h.c1) / (sqrtf(vi / h.c2) + h.eps) + h.wd * wi);
        w[i] = wi;
      }
      const __nv_bfloat16 b = __float2bfloat16_rn(wi);
      wb[i] = b;
      tile[rr][threadIdx.x] = b;
    }
  }
  __syncthreads();
  for (int cc = threadIdx.y; cc < 32; cc += 8) {
    const int col = blockIdx.x * 32 + cc, r = blockIdx.y * 32 + threadIdx.x;
    if (col < k && r < n) wt[static_cast<size_t>(col) * n + r] = tile[threadIdx.x][cc];
  }
}

__global__ void adamw_vec_kernel(Adam h, int n, float* w, float* m, float* v, const float* g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = h.beta1 * m[i] + (1.0f - h.beta1) * gi;
  const float vi = h.beta2 * v[i] + (1.0f - h.beta2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] = w[i] - h.lr * ((mi / h.c1) / (sqrtf(vi / h.c2) + h.eps) + h.wd * w[i]);
}

__global__ void init_kernel(uint64_t seed, int n, int k, int nvalid, float gain, float* w) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<size_t>(n) * k) return;
  const int r = static_cast<int>(i / k);
  const float a = gain * sqrtf(3.0f / static_cast<float>(k));
  w[i] = r < nvalid ? static_cast<float>((2.0 * uniform(seed, i, 77) - 1.0) * a) : 0.0f;
}

// ------------------------------------------------------------------------------- the FP64 DIA

__global__ void dia_f64_kernel(DiaF64 t, int npts, const float* __restrict__ a,
                               const float* __restrict__ cg, const float* __restrict__ kdm,
                               const float* __restrict__ sc, double* __restrict__ stats,
                               double* __restrict__ s64, double* __restrict__ d64) {
  extern __shared__ double dsm[];
  __shared__ double red[32];
  const int ip = blockIdx.x, tid = threadIdx.x, nb = blockDim.x;
  const int nth = t.nth, nfr = t.nfr, nspec = t.nspec, nspecx = t.nspecx, nk = t.nk;
  const int nspecy = t.nfrhgh * nth;
  double* const ue = dsm;
  double* arr[8];
  for (int j = 0; j < 8; ++j) arr[j] = ue + (nspecy + nth) + static_cast<size_t>(j) * (nspecx + nth);
  double* const sa1 = arr[0];
  double* const sa2 = arr[1];
  double* const da1c = arr[2];
  double* const da1p = arr[3];
  double* const da1m = arr[4];
  double* const da2c = arr[5];
  double* const da2p = arr[6];
  double* const da2m = arr[7];
  double* const conx = arr[7] + (nspecx + nth);  // nk
  double* const rowr = conx + nk;                // nk: band tendency of the FP64 S
  double* const rowc = rowr + nk;                // nk: band tendency of the candidate
  const double tpiinv = 1.0 / (2.0 * kPi);

  // 1. CONS (snl1_team.hpp:383-390), MAX(a, b) as (a < b) ? b : a.
  const double kd = kdm[ip];
  const double x0 = t.kdcon * kd;
  const double x = x0 < t.kdmn ? t.kdmn : x0;
  const double y0 = t.snls3 * x;
  const double x2 = -1.e15 < y0 ? y0 : -1.e15;
  const double cons = t.snlc1 * (1.0 + t.snls1 / x * (1.0 - t.snls2 * x) * exp(x2));

  // 2. UE = A / CONX, the zero bins and the parametric tail (:392-426).
  const float* ap = a + static_cast<size_t>(ip) * nspec;
  for (int k = tid; k < nk; k += nb) {
    conx[k] = tpiinv / t.sig[k] * static_cast<double>(cg[static_cast<size_t>(ip) * nk + k]);
    rowr[k] = 0.0;
    rowc[k] = 0.0;
  }
  for (int i = tid; i < nth; i += nb) {
    ue[i] = 0.0;
    for (int j = 0; j < 8; ++j) arr[j][i] = 0.0;
  }
  __syncthreads();
  for (int i = tid; i < nspec; i += nb) ue[i + nth] = static_cast<double>(ap[i]) / conx[i / nth];
  __syncthreads();
  for (int ifr = nfr; ifr < t.nfrhgh; ++ifr) {
    for (int i = tid; i < nth; i += nb) ue[ifr * nth + i + nth] = ue[ifr * nth + i] * t.fachfe;
    __syncthreads();
  }

  // 3. Interactions over the extended spectrum (:433-473), through the index tables.
  for (int isp = tid; isp < nspecx; isp += nb) {
    auto U = [&](int j) { return ue[t.ipim[static_cast<size_t>(j) * nspecx + isp] + nth]; };
    const double e00 = ue[isp + nth];
    const double ep1 = t.awg[0] * U(0) + t.awg[1] * U(1) + t.awg[2] * U(2) + t.awg[3] * U(3);
    const double em1 = t.awg[4] * U(4) + t.awg[5] * U(5) + t.awg[6] * U(6) + t.awg[7] * U(7);
    const double ep2 = t.awg[0] * U(8) + t.awg[1] * U(9) + t.awg[2] * U(10) + t.awg[3] * U(11);
    const double em2 = t.awg[4] * U(12) + t.awg[5] * U(13) + t.awg[6] * U(14) + t.awg[7] * U(15);
    const double af = t.af11[isp / nth];
    const double factor = cons * af * e00;
    const double sa1a = e00 * (ep1 * t.dal1 + em1 * t.dal2);
    const double sa1b = sa1a - ep1 * em1 * t.dal3;
    const double sa2a = e00 * (ep2 * t.dal1 + em2 * t.dal2);
    const double sa2b = sa2a - ep2 * em2 * t.dal3;
    sa1[isp + nth] = factor * sa1b;
    sa2[isp + nth] = factor * sa2b;
    da1c[isp + nth] = cons * af * (sa1a + sa1b);
    da1p[isp + nth] = factor * (t.dal1 * e00 - t.dal3 * em1);
    da1m[isp + nth] = factor * (t.dal2 * e00 - t.dal3 * ep1);
    da2c[isp + nth] = cons * af * (sa2a + sa2b);
    da2p[isp + nth] = factor * (t.dal1 * e00 - t.dal3 * em2);
    da2m[isp + nth] = factor * (t.dal2 * e00 - t.dal3 * ep2);
  }
  __syncthreads();

  // 4. S and D (:475-496), and the candidate's error terms bin by bin.
  const double xfr = t.xfr;
  double m0 = 0, m1 = 0, ts = 0, tc = 0, tg = 0, ss = 0, sc1 = 0, e2 = 0, r2 = 0;
  for (int isp = tid; isp < nspec; isp += nb) {
    auto C1 = [&](int j) { return t.ic[static_cast<size_t>(j) * nspec + isp] + nth; };
    auto C2 = [&](int j) { return t.ic[static_cast<size_t>(8 + j) * nspec + isp] + nth; };
    const int k = isp / nth;
    double acc = -2.0 * (sa1[isp + nth] + sa2[isp + nth]);
    double dac = -2.0 * (da1c[isp + nth] + da2c[isp + nth]);
    for (int j = 0; j < 8; ++j) {
      acc += t.awg[j] * (sa1[C1(j)] + sa2[C2(j)]);
      dac += t.swg[j] * (j < 4 ? (da1p[C1(j)] + da2p[C2(j)]) : (da1m[C1(j)] + da2m[C2(j)]));
    }
    const double sv = conx[k] * acc;
    if (s64) s64[static_cast<size_t>(ip) * nspec + isp] = sv;
    if (d64) d64[static_cast<size_t>(ip) * nspec + isp] = dac;
    const double sig = t.sig[k];
    const double dden = t.dth * (0.5 * sig * (xfr - 1.0 / xfr)) * sig;
    const double w = dden / static_cast<double>(cg[static_cast<size_t>(ip) * nk + k]);
    const double av = ap[isp];
    const double cv = sc ? static_cast<double>(sc[static_cast<size_t>(ip) * nspec + isp]) : 0.0;
    m0 += w * av;
    m1 += w * sig * av;
    ts += w * sv;
    tc += w * cv;
    tg += w * fabs(sv);
    ss += w * sig * sv;
    sc1 += w * sig * cv;
    e2 += (cv - sv) * (cv - sv);
    r2 += sv * sv;
    atomicAdd(rowr + k, w * sv);
    atomicAdd(rowc + k, w * cv);
  }
  m0 = block_sum(m0, red);
  m1 = block_sum(m1, red);
  ts = block_sum(ts, red);
  tc = block_sum(tc, red);
  tg = block_sum(tg, red);
  ss = block_sum(ss, red);
  sc1 = block_sum(sc1, red);
  e2 = block_sum(e2, red);
  r2 = block_sum(r2, red);
  if (tid == 0) {
    double bn = 0, bd = 0;
    for (int k = 0; k < nk; ++k) {
      bn += fabs(rowc[k] - rowr[k]);
      bd += fabs(rowr[k]);
    }
    const double hs = 4.0 * sqrt(m0 > 0 ? m0 : 0.0);
    const double f = hs > 0 ? 8.0 / hs : 0.0;
    double* o = stats + static_cast<size_t>(ip) * 10;
    o[0] = hs;
    o[1] = f * ts;
    o[2] = f * tc;
    o[3] = f * tg;
    o[4] = f * bn;
    o[5] = f * bd;
    o[6] = e2;
    o[7] = r2;
    o[8] = m0 > 0 ? (ss * m0 - m1 * ts) / (m0 * m0) : 0.0;
    o[9] = m0 > 0 ? (sc1 * m0 - m1 * tc) / (m0 * m0) : 0.0;
  }
}

inline dim3 grid1(long long n) { return dim3(static_cast<unsigned>(n)); }

}  // namespace

void synth(const SurGrid& g, const SynthDraw& d, long long p0, int npts, float* a, float* cg,
           float* kdmean, cudaStream_t st) {
  if (npts <= 0) return;
  if (g.nk > 64 || g.nth > 64) throw CudaError(cudaErrorInvalidValue, "synth: NK or NTH above 64");
  synth_kernel<<<grid1(npts), 64, 0, st>>>(g, d, p0, npts, a, cg, kdmean);
  WWB_CHECK(cudaGetLastError());
}

void prep(const SurGrid& g, int npts, const float* a, const float* cg, const float* kdmean,
          __nv_bfloat16* x, int ldx, float* ps, int* shift, cudaStream_t st, float* dzero,
          float* gzero) {
  if (npts <= 0) return;
  if (g.nk > 64) throw CudaError(cudaErrorInvalidValue, "prep: NK above 64");
  const size_t smem =
      static_cast<size_t>(kPointsPerCta) * prep_floats(g.nspec, g.nk, g.nth) * sizeof(float);
  static size_t set = 48 * 1024;
  if (smem > set) {
    WWB_CHECK(cudaFuncSetAttribute(prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    set = smem;
  }
  const unsigned blocks = static_cast<unsigned>((npts + kPointsPerCta - 1) / kPointsPerCta);
  // 36 x 36 with 16-byte aligned spectra and 8-byte aligned input rows: rows across lanes.
  const bool rows36 = g.nk == 36 && g.nth == 36 && g.nspec == 1296 &&
                      (reinterpret_cast<uintptr_t>(a) & 15u) == 0 &&
                      (reinterpret_cast<uintptr_t>(x) & 7u) == 0 && ldx % 4 == 0 &&
                      (reinterpret_cast<uintptr_t>(dzero) & 15u) == 0;
  if (rows36) {
    prep_rows_kernel<36, 36><<<blocks, 32 * kPointsPerCta, 0, st>>>(g, npts, a, cg, kdmean, x,
                                                                     ldx, ps, shift, dzero, gzero);
    WWB_CHECK(cudaGetLastError());
    return;
  }
  prep_kernel<<<blocks, 32 * kPointsPerCta, smem, st>>>(g, npts, a, cg, kdmean, x, ldx, ps,
                                                         shift, dzero, gzero);
  WWB_CHECK(cudaGetLastError());
}

void rowscale_acc(const SurGrid& g, int npts, const float* s, const float* ps, double* acc,
                  unsigned long long* cnt, cudaStream_t st) {
  if (npts <= 0) return;
  if (g.nk > 64) throw CudaError(cudaErrorInvalidValue, "rowscale: NK above 64");
  rowscale_kernel<<<grid1(npts), kThreads, 0, st>>>(g, npts, s, ps, acc, cnt);
  WWB_CHECK(cudaGetLastError());
}

void targets(const SurGrid& g, int npts, const float* s, const float* ps, const int* shift,
             float* t, int ldt, cudaStream_t st) {
  if (npts <= 0) return;
  targets_kernel<<<grid1(npts), kThreads, 0, st>>>(g, npts, s, ps, shift, t, ldt);
  WWB_CHECK(cudaGetLastError());
}

namespace {

__global__ void gather_rows_kernel(const int* __restrict__ count, const int* __restrict__ rows,
                                   int cap, int width, const float* __restrict__ src,
                                   float* __restrict__ dst, int* __restrict__ list_dst,
                                   int* __restrict__ count_dst) {
  const int n = *count;
  const int m = n < cap ? n : cap;
  if (blockIdx.x == 0 && threadIdx.x == 0) *count_dst = n;
  for (int i = blockIdx.x; i < m; i += gridDim.x) {
    const int r = rows[i];
    if (threadIdx.x == 0) list_dst[i] = r;
    const float4* s4 = reinterpret_cast<const float4*>(src + static_cast<size_t>(r) * width);
    float4* d4 = reinterpret_cast<float4*>(dst + static_cast<size_t>(i) * width);
    for (int j = threadIdx.x; j < width / 4; j += blockDim.x) d4[j] = s4[j];
  }
}
}  // namespace

void gate_points(const GateParams& gate, int npts, const float* gsum, const float* head,
                 int* accepted, float* gv, int* rej_list, int* nrej, int* nrej_total,
                 cudaStream_t st, int base) {
  if (npts <= 0) return;
  gate_kernel<<<(npts + 255) / 256, 256, 0, st>>>(gate, npts, gsum, head, accepted, gv, rej_list,
                                                  nrej, nrej_total, base);
  WWB_CHECK(cudaGetLastError());
}

void loss_grad(const SurGrid& g, const LossWeights& w, int m, int nvalid, const float* out,
               int ldo, const float* t, int ldt, const float* ps, __nv_bfloat16* grad, int ldg,
               float* loss, cudaStream_t st) {
  if (m <= 0) return;
  if (ps != nullptr && g.nk > 64) throw CudaError(cudaErrorInvalidValue, "loss: NK above 64");
  loss_kernel<<<grid1(m), kThreads, 0, st>>>(g, w, m, nvalid, out, ldo, t, ldt, ps, grad, ldg,
                                             loss);
  WWB_CHECK(cudaGetLastError());
}

void gather_batch(int m, long long n, uint64_t seed, long long offset, const __nv_bfloat16* xs,
                  int ldx, const float* ts, int ldt, const float* pss, int ldp,
                  __nv_bfloat16* xb, float* tb, float* psb, cudaStream_t st) {
  if (m <= 0) return;
  if (ldx % 8 || ldt % 4) throw CudaError(cudaErrorInvalidValue, "gather: unaligned rows");
  gather_kernel<<<grid1(m), 128, 0, st>>>(m, n, seed, offset, xs, ldx, ts, ldt, pss, ldp, xb, tb,
                                          psb);
  WWB_CHECK(cudaGetLastError());
}

void transpose(const __nv_bfloat16* src, int rows, int cols, int lds, __nv_bfloat16* dst, int ldd,
               cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return;
  const dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_kernel<<<grid, block, 0, st>>>(src, rows, cols, lds, dst, ldd);
  WWB_CHECK(cudaGetLastError());
}

void colsum(const __nv_bfloat16* gt, int n, int m, int ldt, float* db, cudaStream_t st) {
  if (n <= 0) return;
  if (m % 8 || ldt % 8) throw CudaError(cudaErrorInvalidValue, "colsum: rows not multiples of 8");
  colsum_kernel<<<(n + 7) / 8, 256, 0, st>>>(gt, n, m, ldt, db);
  WWB_CHECK(cudaGetLastError());
}

void adamw(const Adam& h, int n, int k, float* w, float* m, float* v, float* g,
           __nv_bfloat16* wb, __nv_bfloat16* wt, cudaStream_t st) {
  const dim3 grid((k + 31) / 32, (n + 31) / 32), block(32, 8);
  adamw_kernel<<<grid, block, 0, st>>>(h, n, k, w, m, v, g, wb, wt, 1);
  WWB_CHECK(cudaGetLastError());
}

void adamw_vec(const Adam& h, int n, float* w, float* m, float* v, const float* g,
               cudaStream_t st) {
  adamw_vec_kernel<<<(n + 255) / 256, 256, 0, st>>>(h, n, w, m, v, g);
  WWB_CHECK(cudaGetLastError());
}

void to_bf16(const float* w, int n, int k, __nv_bfloat16* wb, __nv_bfloat16* wt, cudaStream_t st) {
  const dim3 grid((k + 31) / 32, (n + 31) / 32), block(32, 8);
  Adam h{};
  adamw_kernel<<<grid, block, 0, st>>>(h, n, k, const_cast<float*>(w), nullptr, nullptr, nullptr,
                                       wb, wt, 0);
  WWB_CHECK(cudaGetLastError());
}

void init_weights(uint64_t seed, int n, int k, int nrows_valid, float gain, float* w,
                  __nv_bfloat16* wb, __nv_bfloat16* wt, cudaStream_t st) {
  const size_t total = static_cast<size_t>(n) * k;
  init_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, st>>>(seed, n, k, nrows_valid,
                                                                          gain, w);
  WWB_CHECK(cudaGetLastError());
  to_bf16(w, n, k, wb, wt, st);
}

size_t dia_f64_smem(const DiaF64& t) {
  const size_t nspecy = static_cast<size_t>(t.nfrhgh) * t.nth;
  return (nspecy + t.nth + 8 * static_cast<size_t>(t.nspecx + t.nth) + 3 * t.nk) * sizeof(double);
}

void dia_f64_judge(const DiaF64& t, int npts, const float* a, const float* cg,
                   const float* kdmean, const float* s_cand, double* stats, double* s64,
                   double* d64, cudaStream_t st) {
  if (npts <= 0) return;
  const size_t smem = dia_f64_smem(t);
  if (smem > 227 * 1024) throw CudaError(cudaErrorInvalidValue, "FP64 DIA: tables too large");
  static size_t set = 0;
  if (smem > set) {
    WWB_CHECK(cudaFuncSetAttribute(dia_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    set = smem;
  }
  dia_f64_kernel<<<grid1(npts), kThreads, smem, st>>>(t, npts, a, cg, kdmean, s_cand, stats, s64,
                                                       d64);
  WWB_CHECK(cudaGetLastError());
}

}  // namespace mlp
}  // namespace wwb

namespace wwb {
namespace mlp {
void gather_listed_rows(const int* count, const int* rows, int cap, int width, const float* src,
                        float* dst, int* list_dst, int* count_dst, cudaStream_t st) {
  if (width % 4 != 0)
    throw CudaError(cudaErrorInvalidValue, "gather_listed_rows: row width not a multiple of 4");
  gather_rows_kernel<<<512, 256, 0, st>>>(count, rows, cap, width, src, dst, list_dst, count_dst);
  WWB_CHECK(cudaGetLastError());
}
}  // namespace mlp
}  // namespace wwb
