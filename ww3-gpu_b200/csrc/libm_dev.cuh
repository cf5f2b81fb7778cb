// ww3-gpu_b200/csrc/libm_dev.cuh
// Float libm for the device with the bits of the host's glibc, where a kernel must reproduce a
// CPU result exactly.
//
// expf: the method of Szabolcs Nagy's expf in ARM's optimized-routines (MIT / Apache-2.0),
// which glibc uses since 2.27 (sysdeps/ieee754/flt-32/e_expf.c): x*N/ln2 = k + r with N = 32,
// 2^(k/N) from a 32-entry table of 2^(i/32) in double, 2^(r/N) by a cubic in double, one final
// rounding to float. The table is 2^(i/32) rounded to double with (i << 47) subtracted from its
// bits, generated from that definition (tests/test_libm.py regenerates it with Python's decimal
// module and compares). On x86-64 glibc runs this source compiled with FMA instructions
// (__expf_fma); which of its multiply-adds are fused is not something this file assumes: it is
// the template argument, and tests/test_libm.py picks the variant that equals this host's glibc
// expf on all 2^32 inputs (the host build of this header uses C's fma(), the device build
// __fma_rn, so both builds compute the same bits).
//
// The reference (ww3-gpu kokkos/src/ww_kokkos/libm_device.hpp:33-52) calls expf in W3SNL1's
// CONS (snl1_team.hpp:386-390); that is the only libm call of the DIA.
#pragma once

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define WWB_HD __host__ __device__ __forceinline__
#else
#include <math.h>
#define WWB_HD inline
#endif

namespace wwb {
namespace dm {

#define WWB_EXP2F_TAB                                                                       \
  {0x3ff0000000000000ULL, 0x3fefd9b0d3158574ULL, 0x3fefb5586cf9890fULL, 0x3fef9301d0125b51ULL, \
   0x3fef72b83c7d517bULL, 0x3fef54873168b9aaULL, 0x3fef387a6e756238ULL, 0x3fef1e9df51fdee1ULL, \
   0x3fef06fe0a31b715ULL, 0x3feef1a7373aa9cbULL, 0x3feedea64c123422ULL, 0x3feece086061892dULL, \
   0x3feebfdad5362a27ULL, 0x3feeb42b569d4f82ULL, 0x3feeab07dd485429ULL, 0x3feea47eb03a5585ULL, \
   0x3feea09e667f3bcdULL, 0x3fee9f75e8ec5f74ULL, 0x3feea11473eb0187ULL, 0x3feea589994cce13ULL, \
   0x3feeace5422aa0dbULL, 0x3feeb737b0cdc5e5ULL, 0x3feec49182a3f090ULL, 0x3feed503b23e255dULL, \
   0x3feee89f995ad3adULL, 0x3feeff76f2fb5e47ULL, 0x3fef199bdd85529cULL, 0x3fef3720dcef9069ULL, \
   0x3fef5818dcfba487ULL, 0x3fef7c97337b9b5fULL, 0x3fefa4afa2a490daULL, 0x3fefd0765b6e4540ULL}

#if defined(__CUDACC__)
__device__ __constant__ static const uint64_t kExp2fTabDev[32] = WWB_EXP2F_TAB;
#endif
static const uint64_t kExp2fTabHost[32] = WWB_EXP2F_TAB;

WWB_HD uint64_t exp2f_tab(unsigned i) {
#if defined(__CUDA_ARCH__)
  return kExp2fTabDev[i];
#else
  return kExp2fTabHost[i];
#endif
}

WWB_HD double fma_d(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}
WWB_HD uint32_t asuint(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}
WWB_HD uint64_t asuint64(double f) {
  uint64_t u;
  memcpy(&u, &f, 8);
  return u;
}
WWB_HD double asdouble(uint64_t u) {
  double f;
  memcpy(&f, &u, 8);
  return f;
}
WWB_HD float asfloat(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}

// Polynomial for 2^(r/N) - 1 with r in [-1/2, 1/2], coefficients of optimized-routines'
// exp2f_data scaled by powers of N = 32; InvLn2N = N / ln 2 rounded to double.
constexpr double kInvLn2N = 0x1.71547652b82fep+0 * 32;
constexpr double kShift = 0x1.8p+52;
constexpr double kC0 = 0x1.c6af84b912394p-5 / 32 / 32 / 32;
constexpr double kC1 = 0x1.ebfce50fac4f3p-3 / 32 / 32;
constexpr double kC2 = 0x1.62e42ff0c52d6p-1 / 32;

/// expf. FUSE bit 0: the rounding shift z + Shift is one fused multiply-add; bit 1: r = z - k
/// is fused with the product z = x * N/ln2; bit 2: the three polynomial steps are fused.
template <int FUSE>
WWB_HD float expf_t(float x) {
  const uint32_t abstop = (asuint(x) >> 20) & 0x7ff;
  if (abstop >= (asuint(88.0f) >> 20)) {
    if (asuint(x) == 0xff800000u) return 0.0f;  // -inf
    if (abstop >= 0x7f8) return x + x;          // +inf, nan
    if (x > 0x1.62e42ep6f) return asfloat(0x7f800000u);  // overflow: +inf
    if (x < -0x1.9fe368p6f) return 0.0f;                 // underflow: +0
  }
  const double xd = (double)x;
  const double z = kInvLn2N * xd;
  double kd = (FUSE & 1) ? fma_d(kInvLn2N, xd, kShift) : z + kShift;
  const uint64_t ki = asuint64(kd);
  kd -= kShift;
  const double r = (FUSE & 2) ? fma_d(kInvLn2N, xd, -kd) : z - kd;
  uint64_t t = exp2f_tab((unsigned)(ki % 32));
  t += ki << (52 - 5);
  const double s = asdouble(t);
  double y;
  if (FUSE & 4) {
    const double p = fma_d(kC0, r, kC1);
    const double r2 = r * r;
    y = fma_d(kC2, r, 1.0);
    y = fma_d(p, r2, y);
  } else {
    const double p = kC0 * r + kC1;
    const double r2 = r * r;
    y = kC2 * r + 1.0;
    y = p * r2 + y;
  }
  y = y * s;
  return (float)y;
}

/// The variant that equals glibc's expf on this platform (tests/test_libm.py checks all 2^32
/// inputs against the host's glibc).
#ifndef WWB_EXPF_FUSE
#define WWB_EXPF_FUSE 7
#endif
WWB_HD float expf(float x) { return expf_t<WWB_EXPF_FUSE>(x); }

}  // namespace dm
}  // namespace wwb
