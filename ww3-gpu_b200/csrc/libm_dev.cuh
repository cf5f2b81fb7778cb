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
// logf, powf: the same library's logf and powf (glibc since 2.28, sysdeps/ieee754/flt-32/e_logf.c,
// e_powf.c): x = 2^k z with z in [0x3f330000, 2*0x3f330000), one of 16 subintervals picked by the
// top mantissa bits, log(z) = log1p(z/c - 1) + log(c) with 1/c from a table and a polynomial in
// double; powf computes log2 that way (5-term polynomial) and 2^(y log2 x) as exp2f does. The
// 16 values 1/c are the published table; log(c) and log2(c) are generated from them
// (-ln(invc), -log2(invc) rounded to double) and tests/test_libm.py regenerates and compares.
// sincosf: the same library's sincosf (s_sincosf.c): |x| < pi/4 direct, |x| < 120 one
// multiply-subtract by pi/2, larger |x| an exact 2/pi fixed-point reduction with a table of 2/pi
// bits (generated from 2/pi), then degree-8 cosine / degree-7 sine polynomials in double.
// tanhf, atan2f, log10f: glibc 2.39 keeps the fdlibm (Sun, freely redistributable) float
// routines s_tanhf.c (through expm1f), e_atan2f.c (through atanf) and e_log10f.c (through logf);
// written here from that published method with its float constants (given as bit patterns).
// exp, tanh in double (W3SDB1): not glibc's bits; exp by a 2^(k/64) split with a degree-7
// Taylor tail in double, tanh from it; they feed double expressions rounded to float afterwards.
//
// The reference (ww3-gpu kokkos/src/ww_kokkos/libm_device.hpp:33-52) calls expf in W3SNL1's
// CONS (snl1_team.hpp:386-390), the ST4 source terms and W3SRCE call the rest
// (st4_sin4.hpp, st4_sds4.hpp, st4_spr4.hpp, srce_kernel.hpp, srce_db1.hpp).
// The device copies of the tables are global-memory arrays read through the read-only cache:
// lanes of a warp index them with different values, which constant memory would serialize.
#pragma once

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define WWB_HD __host__ __device__ __forceinline__
// The public functions are called, not inlined: a kernel that calls them from dozens of sites
// stays small enough for the instruction cache when several CTAs run different phases.
#define WWB_HC static __host__ __device__ __noinline__
#else
#include <math.h>
#define WWB_HD inline
#define WWB_HC inline
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
__device__ static const uint64_t kExp2fTabDev[32] = WWB_EXP2F_TAB;
#endif
static const uint64_t kExp2fTabHost[32] = WWB_EXP2F_TAB;

#if defined(__CUDA_ARCH__)
/// Table loads through the read-only path, kept in L1 ahead of streamed data (evict_last): the
/// tables are a few KB, and a serial chain pays an L2 round trip for every miss.
__device__ __forceinline__ uint64_t tab_ld64(const void* p) {
  uint64_t v;
  asm("ld.global.nc.L1::evict_last.b64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ uint32_t tab_ld32(const void* p) {
  uint32_t v;
  asm("ld.global.nc.L1::evict_last.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
#endif

WWB_HD uint64_t exp2f_tab(unsigned i) {
#if defined(__CUDA_ARCH__)
  return tab_ld64(&kExp2fTabDev[i]);
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
WWB_HC float expf(float x) { return expf_t<WWB_EXPF_FUSE>(x); }

WWB_HD float fma_f(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}

// ------------------------------------------------------------------------------------ logf
// 1/c of the 16 subintervals (published table of the method).
#define WWB_LOG_INVC                                                                          \
  {0x1.661ec79f8f3bep+0, 0x1.571ed4aaf883dp+0, 0x1.49539f0f010bp+0, 0x1.3c995b0b80385p+0,     \
   0x1.30d190c8864a5p+0, 0x1.25e227b0b8eap+0, 0x1.1bb4a4a1a343fp+0, 0x1.12358f08ae5bap+0,     \
   0x1.0953f419900a7p+0, 0x1p+0, 0x1.e608cfd9a47acp-1, 0x1.ca4b31f026aap-1,                 \
   0x1.b2036576afce6p-1, 0x1.9c2d163a1aa2dp-1, 0x1.886e6037841edp-1, 0x1.767dcf5534862p-1}
// ln(c) = -ln(invc) rounded to double (generated; checked by tests/test_libm.py).
#define WWB_LOG_LOGC                                                                          \
  {-0x1.57bf7808caadep-2, -0x1.2bef0a7c06ddbp-2, -0x1.01eae7f513a67p-2, -0x1.b31d8a68224e9p-3, \
   -0x1.6574f0ac07758p-3, -0x1.1aa2bc79c81p-3, -0x1.a4e76ce8c0e5ep-4, -0x1.1973c5a611cccp-4,  \
   -0x1.252f438e10c1ep-5, 0x0p+0, 0x1.aa5aa5df25984p-5, 0x1.c5e53aa362eb4p-4,                 \
   0x1.526e57720db08p-3, 0x1.bc2860d22477p-3, 0x1.1058bc8a07ee1p-2, 0x1.4043057b6ee09p-2}
// log2(c) = -log2(invc) rounded to double (generated; checked by tests/test_libm.py).
#define WWB_LOG2_LOGC                                                                         \
  {-0x1.efec65b963019p-2, -0x1.b0b6832d4fca4p-2, -0x1.7418b0a1fb77bp-2, -0x1.39de91a6dcf7bp-2, \
   -0x1.01d9bf3f2b631p-2, -0x1.97c1d1b3b7afp-3, -0x1.2f9e393af3c9fp-3, -0x1.960cbbf788d5cp-4,  \
   -0x1.a6f9db6475fcep-5, 0x0p+0, 0x1.338ca9f24f53dp-4, 0x1.476a9543891bap-3,                 \
   0x1.e840b4ac4e4d2p-3, 0x1.40645f0c6651cp-2, 0x1.88e9c2c1b9ff8p-2, 0x1.ce0a44eb17bccp-2}

#if defined(__CUDACC__)
__device__ static const double kLogInvcDev[16] = WWB_LOG_INVC;
__device__ static const double kLogLogcDev[16] = WWB_LOG_LOGC;
__device__ static const double kLog2LogcDev[16] = WWB_LOG2_LOGC;
#endif
static const double kLogInvcHost[16] = WWB_LOG_INVC;
static const double kLogLogcHost[16] = WWB_LOG_LOGC;
static const double kLog2LogcHost[16] = WWB_LOG2_LOGC;

WWB_HD double log_invc(unsigned i) {
#if defined(__CUDA_ARCH__)
  return asdouble(tab_ld64(&kLogInvcDev[i]));
#else
  return kLogInvcHost[i];
#endif
}
WWB_HD double log_logc(unsigned i) {
#if defined(__CUDA_ARCH__)
  return asdouble(tab_ld64(&kLogLogcDev[i]));
#else
  return kLogLogcHost[i];
#endif
}
WWB_HD double log2_logc(unsigned i) {
#if defined(__CUDA_ARCH__)
  return asdouble(tab_ld64(&kLog2LogcDev[i]));
#else
  return kLog2LogcHost[i];
#endif
}

constexpr uint32_t kLogOff = 0x3f330000u;
constexpr double kLn2 = 0x1.62e42fefa39efp-1;
// log1p(r) ~ r + A0 r^2 + A1 r^3 + A2 r^4 (published coefficients of the method).
constexpr double kLogA0 = -0x1.00ea348b88334p-2, kLogA1 = 0x1.5575b0be00b6ap-2,
                 kLogA2 = -0x1.ffffef20a4123p-2;

/// Multiply-add, fused or not (the FMA build of glibc contracts a*b+c).
template <bool F>
WWB_HD double madd(double a, double b, double c) {
  return F ? fma_d(a, b, c) : a * b + c;
}

/// logf. FUSE bit 0: r = z*invc - 1 fused; bit 1: y0 = logc + k*Ln2 fused; bit 2: the three
/// polynomial steps fused.
template <int FUSE>
WWB_HD float logf_t(float x) {
  uint32_t ix = asuint(x);
  if (ix == 0x3f800000u) return 0.0f;
  if (ix - 0x00800000u >= 0x7f800000u - 0x00800000u) {
    if (ix * 2 == 0) return asfloat(0xff800000u);                  // log(+-0) = -inf
    if (ix == 0x7f800000u) return x;                               // log(inf) = inf
    if ((ix & 0x80000000u) || ix * 2 >= 0xff000000u) return (x - x) / (x - x);  // nan
    ix = asuint(x * 0x1p23f);                                      // subnormal
    ix -= 23u << 23;
  }
  const uint32_t tmp = ix - kLogOff;
  const unsigned i = (tmp >> (23 - 4)) % 16;
  const int k = (int32_t)tmp >> 23;
  const uint32_t iz = ix - (tmp & 0xff800000u);
  const double invc = log_invc(i), logc = log_logc(i);
  const double z = (double)asfloat(iz);
  const double r = madd<(FUSE & 1) != 0>(z, invc, -1.0);
  const double y0 = madd<(FUSE & 2) != 0>((double)k, kLn2, logc);
  const double r2 = r * r;
  double y = madd<(FUSE & 4) != 0>(kLogA1, r, kLogA2);
  y = madd<(FUSE & 4) != 0>(kLogA0, r2, y);
  y = madd<(FUSE & 4) != 0>(y, r2, y0 + r);
  return (float)y;
}
#ifndef WWB_LOGF_FUSE
#define WWB_LOGF_FUSE 7
#endif
WWB_HC float logf(float x) { return logf_t<WWB_LOGF_FUSE>(x); }

// ------------------------------------------------------------------------------------ powf
// log1p(r)/ln2 ~ A0 r^5 + A1 r^4 + A2 r^3 + A3 r^2 + A4 r (published coefficients).
constexpr double kPowA0 = 0x1.27616c9496e0bp-2, kPowA1 = -0x1.71969a075c67ap-2,
                 kPowA2 = 0x1.ec70a6ca7baddp-2, kPowA3 = -0x1.7154748bef6c8p-1,
                 kPowA4 = 0x1.71547652ab82bp0;
// 2^r ~ C0 r^3 + C1 r^2 + C2 r + 1 for |r| <= 1/64 (the exp2f coefficients, unscaled).
constexpr double kExp2C0 = 0x1.c6af84b912394p-5, kExp2C1 = 0x1.ebfce50fac4f3p-3,
                 kExp2C2 = 0x1.62e42ff0c52d6p-1;
constexpr double kExp2Shift = 0x1.8p+52 / 32;

template <int FUSE>
WWB_HD double pow_log2(uint32_t ix) {
  const uint32_t tmp = ix - kLogOff;
  const unsigned i = (tmp >> (23 - 4)) % 16;
  const uint32_t top = tmp & 0xff800000u;
  const uint32_t iz = ix - top;
  const int k = (int32_t)top >> 23;
  const double invc = log_invc(i), logc = log2_logc(i);
  const double z = (double)asfloat(iz);
  const double r = madd<(FUSE & 1) != 0>(z, invc, -1.0);
  const double y0 = logc + (double)k;
  const double r2 = r * r;
  double y = madd<(FUSE & 2) != 0>(kPowA0, r, kPowA1);
  const double p = madd<(FUSE & 2) != 0>(kPowA2, r, kPowA3);
  const double r4 = r2 * r2;
  double q = madd<(FUSE & 2) != 0>(kPowA4, r, y0);
  q = madd<(FUSE & 2) != 0>(p, r2, q);
  y = madd<(FUSE & 2) != 0>(y, r4, q);
  return y;
}

template <int FUSE>
WWB_HD float pow_exp2(double xd, uint32_t sign_bias) {
  double kd = xd + kExp2Shift;
  const uint64_t ki = asuint64(kd);
  kd -= kExp2Shift;
  const double r = xd - kd;
  uint64_t t = exp2f_tab((unsigned)(ki % 32));
  const uint64_t ski = ki + sign_bias;
  t += ski << (52 - 5);
  const double s = asdouble(t);
  const double z = madd<(FUSE & 4) != 0>(kExp2C0, r, kExp2C1);
  const double r2 = r * r;
  double y = madd<(FUSE & 4) != 0>(kExp2C2, r, 1.0);
  y = madd<(FUSE & 4) != 0>(z, r2, y);
  y = y * s;
  return (float)y;
}

/// 0: y not an integer, 1: odd integer, 2: even integer.
WWB_HD int pow_checkint(uint32_t iy) {
  const int e = iy >> 23 & 0xff;
  if (e < 0x7f) return 0;
  if (e > 0x7f + 23) return 2;
  if (iy & ((1u << (0x7f + 23 - e)) - 1)) return 0;
  if (iy & (1u << (0x7f + 23 - e))) return 1;
  return 2;
}
WWB_HD bool pow_zeroinfnan(uint32_t i) { return 2 * i - 1 >= 2u * 0x7f800000u - 1; }
WWB_HD bool pow_signaling(uint32_t i) { return 2 * (i ^ 0x00400000u) > 2u * 0x7fc00000u; }

/// powf. FUSE bit 0: r = z*invc - 1 fused; bit 1: the log2 polynomial fused; bit 2: the exp2
/// polynomial fused.
template <int FUSE>
WWB_HD float powf_t(float x, float y) {
  uint32_t sign_bias = 0;
  uint32_t ix = asuint(x);
  const uint32_t iy = asuint(y);
  if (ix - 0x00800000u >= 0x7f800000u - 0x00800000u || pow_zeroinfnan(iy)) {
    if (pow_zeroinfnan(iy)) {
      if (2 * iy == 0) return pow_signaling(ix) ? x + y : 1.0f;
      if (ix == 0x3f800000u) return pow_signaling(iy) ? x + y : 1.0f;
      if (2 * ix > 2u * 0x7f800000u || 2 * iy > 2u * 0x7f800000u) return x + y;
      if (2 * ix == 2 * 0x3f800000u) return 1.0f;
      if ((2 * ix < 2 * 0x3f800000u) == !(iy & 0x80000000u)) return 0.0f;
      return y * y;
    }
    if (pow_zeroinfnan(ix)) {
      float x2 = x * x;
      if ((ix & 0x80000000u) && pow_checkint(iy) == 1) x2 = -x2;
      return (iy & 0x80000000u) ? 1.0f / x2 : x2;
    }
    if (ix & 0x80000000u) {
      const int yint = pow_checkint(iy);
      if (yint == 0) return (x - x) / (x - x);
      if (yint == 1) sign_bias = 1u << (5 + 11);
      ix &= 0x7fffffffu;
    }
    if (ix < 0x00800000u) {
      ix = asuint(x * 0x1p23f);
      ix &= 0x7fffffffu;
      ix -= 23u << 23;
    }
  }
  const double logx = pow_log2<FUSE>(ix);
  const double ylogx = (double)y * logx;
  if ((asuint64(ylogx) >> 47 & 0xffff) >= asuint64(126.0) >> 47) {
    if (ylogx > 0x1.fffffffd1d571p+6)
      return sign_bias ? asfloat(0xff800000u) : asfloat(0x7f800000u);
    if (ylogx <= -150.0) return sign_bias ? -0.0f : 0.0f;
  }
  return pow_exp2<FUSE>(ylogx, sign_bias);
}
#ifndef WWB_POWF_FUSE
#define WWB_POWF_FUSE 7
#endif
WWB_HC float powf(float x, float y) { return powf_t<WWB_POWF_FUSE>(x, y); }

// --------------------------------------------------------------------------------- sincosf
// Cosine 1 + c1 x^2 + ... (c0 = 1) and sine x + s1 x^3 + s2 x^5 + s3 x^7 coefficients of the
// published method; the second set (quadrants 2, 3) negates the cosine.
constexpr double kScC1 = -0x1.ffffffd0c621cp-2, kScC2 = 0x1.55553e1068f19p-5,
                 kScC3 = -0x1.6c087e89a359dp-10, kScC4 = 0x1.99343027bf8c3p-16,
                 kScS1 = -0x1.555545995a603p-3, kScS2 = 0x1.1107605230bc4p-7,
                 kScS3 = -0x1.994eb3774cf24p-13;
constexpr double kHpiInv24 = 0x1.45f306dc9c883p+23;  // 2/pi * 2^24
constexpr double kHpi = 0x1.921fb54442d18p+0;         // pi/2
constexpr double kPio4 = 0x1.921fb54442d18p-1;        // pi/4
constexpr double kPi63 = 0x1.921fb54442d18p-62;       // pi * 2^-63
// 32-bit windows, 8 bits apart, of the binary fraction of 2/pi (generated; checked by
// tests/test_libm.py).
#define WWB_INV_PIO4                                                                     \
  {0xa2u, 0xa2f9u, 0xa2f983u, 0xa2f9836eu, 0xf9836e4eu, 0x836e4e44u, 0x6e4e4415u,         \
   0x4e441529u, 0x441529fcu, 0x1529fc27u, 0x29fc2757u, 0xfc2757d1u, 0x2757d1f5u,         \
   0x57d1f534u, 0xd1f534ddu, 0xf534ddc0u, 0x34ddc0dbu, 0xddc0db62u, 0xc0db6295u,         \
   0xdb629599u, 0x6295993cu, 0x95993c43u, 0x993c4390u, 0x3c439041u}
#if defined(__CUDACC__)
__device__ static const uint32_t kInvPio4Dev[24] = WWB_INV_PIO4;
#endif
static const uint32_t kInvPio4Host[24] = WWB_INV_PIO4;
WWB_HD uint32_t inv_pio4(unsigned i) {
#if defined(__CUDA_ARCH__)
  return tab_ld32(&kInvPio4Dev[i]);
#else
  return kInvPio4Host[i];
#endif
}

WWB_HD uint32_t abstop12(float x) { return (asuint(x) >> 20) & 0x7ff; }

/// The polynomials on the reduced argument; quadrant n odd swaps sine and cosine, `neg` is the
/// second coefficient set (negated cosine).
template <int FUSE>
WWB_HD void sincosf_poly(double x, double x2, bool neg, int n, float* sinp, float* cosp) {
  constexpr bool F = (FUSE & 1) != 0;
  const double c0 = neg ? -1.0 : 1.0, c1 = neg ? -kScC1 : kScC1, c2 = neg ? -kScC2 : kScC2,
               c3 = neg ? -kScC3 : kScC3, c4 = neg ? -kScC4 : kScC4;
  const double x4 = x2 * x2;
  const double x3 = x2 * x;
  const double cc2 = madd<F>(x2, c4, c3);
  const double ss1 = madd<F>(x2, kScS3, kScS2);
  float* const sp = (n & 1) ? cosp : sinp;
  float* const cp = (n & 1) ? sinp : cosp;
  const double cc1 = madd<F>(x2, c1, c0);
  const double x5 = x3 * x2;
  const double x6 = x4 * x2;
  const double s = madd<F>(x3, kScS1, x);
  const double c = madd<F>(x4, c2, cc1);
  *sp = (float)madd<F>(x5, ss1, s);
  *cp = (float)madd<F>(x6, cc2, c);
}

/// sincosf. FUSE bit 0: the polynomial steps fused; bit 1: x - n*pi/2 fused.
template <int FUSE>
WWB_HD void sincosf_t(float y, float* sinp, float* cosp) {
  double x = y;
  if (abstop12(y) < abstop12((float)kPio4)) {
    const double x2 = x * x;
    if (abstop12(y) < abstop12(0x1p-12f)) {
      *sinp = y;
      *cosp = 1.0f;
      return;
    }
    sincosf_poly<FUSE>(x, x2, false, 0, sinp, cosp);
  } else if (abstop12(y) < abstop12(120.0f)) {
    const double r = x * kHpiInv24;
    const int n = ((int32_t)r + 0x800000) >> 24;
    x = (FUSE & 2) ? fma_d(-(double)n, kHpi, x) : x - n * kHpi;
    const double s = (n & 3) == 0 || (n & 3) == 3 ? 1.0 : -1.0;
    sincosf_poly<FUSE>(x * s, x * x, (n & 2) != 0, n, sinp, cosp);
  } else if (abstop12(y) < abstop12(asfloat(0x7f800000u))) {
    uint32_t xi = asuint(y);
    const int sign = xi >> 31;
    const unsigned base = (xi >> 26) & 15;
    const int shift = (xi >> 23) & 7;
    xi = (xi & 0xffffff) | 0x800000;
    xi <<= shift;
    uint64_t res0 = (uint64_t)(uint32_t)(xi * inv_pio4(base));
    const uint64_t res1 = (uint64_t)xi * inv_pio4(base + 4);
    const uint64_t res2 = (uint64_t)xi * inv_pio4(base + 8);
    res0 = (res2 >> 32) | (res0 << 32);
    res0 += res1;
    const uint64_t nn = (res0 + (1ULL << 61)) >> 62;
    res0 -= nn << 62;
    const double xr = (double)(int64_t)res0 * kPi63;
    const int n = (int)nn;
    const int q = (n + sign) & 3;
    const double s = q == 0 || q == 3 ? 1.0 : -1.0;
    sincosf_poly<FUSE>(xr * s, xr * xr, (q & 2) != 0, n, sinp, cosp);
  } else {
    *sinp = *cosp = y - y;
  }
}
#ifndef WWB_SINCOSF_FUSE
#define WWB_SINCOSF_FUSE 3
#endif
WWB_HC void sincosf(float x, float* s, float* c) { sincosf_t<WWB_SINCOSF_FUSE>(x, s, c); }

// ------------------------------------------------------------------------------ expm1f, tanhf
/// fdlibm expm1f (float, no fused operations).
WWB_HD float expm1f(float x) {
  const float one = 1.0f, huge = 1.0e30f, tiny = 1.0e-30f;
  const float o_threshold = asfloat(0x42b17180u), ln2_hi = asfloat(0x3f317180u),
              ln2_lo = asfloat(0x3717f7d1u), invln2 = asfloat(0x3fb8aa3bu);
  const float Q1 = asfloat(0xbd088889u), Q2 = asfloat(0x3ad00d01u), Q3 = asfloat(0xb8a670cdu),
              Q4 = asfloat(0x36867e54u), Q5 = asfloat(0xb457edbbu);
  float y, hi, lo, c = 0.0f, t, e, hxs, hfx, r1;
  int32_t k;
  uint32_t hx = asuint(x);
  const uint32_t xsb = hx & 0x80000000u;
  y = xsb == 0 ? x : -x;
  (void)y;
  hx &= 0x7fffffffu;
  if (hx >= 0x4195b844u) {
    if (hx >= 0x42b17218u) {
      if (hx > 0x7f800000u) return x + x;
      if (hx == 0x7f800000u) return xsb == 0 ? x : -1.0f;
      if (x > o_threshold) return asfloat(0x7f800000u);
    }
    if (xsb != 0) return tiny - one;
  }
  if (hx > 0x3eb17218u) {
    if (hx < 0x3F851592u) {
      if (xsb == 0) {
        hi = x - ln2_hi;
        lo = ln2_lo;
        k = 1;
      } else {
        hi = x + ln2_hi;
        lo = -ln2_lo;
        k = -1;
      }
    } else {
      k = (int32_t)(invln2 * x + (xsb == 0 ? 0.5f : -0.5f));
      t = (float)k;
      hi = x - t * ln2_hi;
      lo = t * ln2_lo;
    }
    x = hi - lo;
    c = (hi - x) - lo;
  } else if (hx < 0x33000000u) {
    t = huge + x;
    return x - (t - (huge + x));
  } else {
    k = 0;
  }
  hfx = 0.5f * x;
  hxs = x * hfx;
  r1 = one + hxs * (Q1 + hxs * (Q2 + hxs * (Q3 + hxs * (Q4 + hxs * Q5))));
  t = 3.0f - r1 * hfx;
  e = hxs * ((r1 - t) / (6.0f - x * t));
  if (k == 0) return x - (x * e - hxs);
  e = (x * (e - c) - c);
  e -= hxs;
  if (k == -1) return 0.5f * (x - e) - 0.5f;
  if (k == 1) {
    if (x < -0.25f) return -2.0f * (e - (x + 0.5f));
    return one + 2.0f * (x - e);
  }
  if (k <= -2 || k > 56) {
    y = one - (e - x);
    if (k == 128) {
      y = y * 2.0f * 0x1p127f;
    } else {
      y = asfloat(asuint(y) + ((uint32_t)k << 23));
    }
    return y - one;
  }
  if (k < 23) {
    t = asfloat(0x3f800000u - (0x1000000u >> k));
    y = t - (e - x);
    y = asfloat(asuint(y) + ((uint32_t)k << 23));
  } else {
    t = asfloat((uint32_t)(0x7f - k) << 23);
    y = x - (e + t);
    y += one;
    y = asfloat(asuint(y) + ((uint32_t)k << 23));
  }
  return y;
}

/// fdlibm tanhf.
WWB_HC float tanhf(float x) {
  const float one = 1.0f, two = 2.0f, tiny = 1.0e-30f;
  const uint32_t jx = asuint(x);
  const uint32_t ix = jx & 0x7fffffffu;
  float t, z;
  if (ix >= 0x7f800000u) {
    if (!(jx & 0x80000000u)) return one / x + one;
    return one / x - one;
  }
  if (ix < 0x41b00000u) {
    if (ix == 0) return x;
    if (ix < 0x24000000u) return x * (one + x);
    if (ix >= 0x3f800000u) {
      t = expm1f(two * fabsf(x));
      z = one - two / (t + two);
    } else {
      t = expm1f(-two * fabsf(x));
      z = -t / (t + two);
    }
  } else {
    z = one - tiny;
  }
  return (jx & 0x80000000u) ? -z : z;
}

// ------------------------------------------------------------------------------ sinhf, coshf
/// sinhf as glibc's e_sinhf.c computes it (fdlibm's method): expm1f below 22, expf up to the
/// overflow threshold.
WWB_HC float sinhf(float x) {
  const float one = 1.0f, shuge = 1.0e37f;
  const uint32_t jx = asuint(x);
  const uint32_t ix = jx & 0x7fffffffu;
  if (ix >= 0x7f800000u) return x + x;
  const float h = (jx & 0x80000000u) ? -0.5f : 0.5f;
  const float ax = fabsf(x);
  if (ix < 0x41b00000u) {  // |x| < 22 (glibc's bound of the expm1f branch)
    if (ix < 0x31800000u) {  // |x| < 2**-28 (glibc's threshold)
      if (shuge + x > one) return x;
    }
    const float t = expm1f(ax);
    if (ix < 0x3f800000u) return h * (2.0f * t - t * t / (t + one));
    return h * (t + t / (t + one));
  }
  if (ix < 0x42b17180u) return h * expf(ax);  // |x| in [22, log(maxfloat)]
  if (ix <= 0x42b2d4fcu) {                   // |x| up to the overflow threshold
    const float w = expf(0.5f * ax);
    const float t = h * w;
    return t * w;
  }
  return x * shuge;
}

/// coshf as glibc's e_coshf.c computes it (fdlibm's method).
WWB_HC float coshf(float x) {
  const float one = 1.0f, half = 0.5f, huge = 1.0e30f;
  const uint32_t ix = asuint(x) & 0x7fffffffu;
  if (ix >= 0x7f800000u) return x * x;
  const float ax = fabsf(x);
  if (ix < 0x3eb17218u) {  // |x| < 0.5*ln2
    const float t = expm1f(ax);
    const float w = one + t;
    if (ix < 0x24000000u) return w;  // cosh(tiny) = 1
    return one + (t * t) / (w + w);
  }
  if (ix < 0x41100000u) {  // |x| < 9
    const float t = expf(ax);
    return half * t + half / t;
  }
  if (ix < 0x42b17180u) return half * expf(ax);
  if (ix <= 0x42b2d4fcu) {
    const float w = expf(half * ax);
    const float t = half * w;
    return t * w;
  }
  return huge * huge;
}

// ----------------------------------------------------------------------------- atanf, atan2f
/// fdlibm atanf.
WWB_HC float atanf(float x) {
  const float one = 1.0f, huge = 1.0e30f;
  const float hi0 = asfloat(0x3eed6338u), hi1 = asfloat(0x3f490fdau), hi2 = asfloat(0x3f7b985eu),
              hi3 = asfloat(0x3fc90fdau);
  const float lo0 = asfloat(0x31ac3769u), lo1 = asfloat(0x33222168u), lo2 = asfloat(0x33140fb4u),
              lo3 = asfloat(0x33a22168u);
  const float T0 = asfloat(0x3eaaaaabu), T1 = asfloat(0xbe4ccccdu), T2 = asfloat(0x3e124925u),
              T3 = asfloat(0xbde38e38u), T4 = asfloat(0x3dba2e6eu), T5 = asfloat(0xbd9d8795u),
              T6 = asfloat(0x3d886b35u), T7 = asfloat(0xbd6ef16bu), T8 = asfloat(0x3d4bda59u),
              T9 = asfloat(0xbd15a221u), T10 = asfloat(0x3c8569d7u);
  const uint32_t hx = asuint(x);
  const uint32_t ix = hx & 0x7fffffffu;
  int id;
  if (ix >= 0x4c000000u) {
    if (ix > 0x7f800000u) return x + x;
    if (!(hx & 0x80000000u)) return hi3 + lo3;
    return -hi3 - lo3;
  }
  if (ix < 0x3ee00000u) {
    if (ix < 0x31000000u) {
      if (huge + x > one) return x;
    }
    id = -1;
  } else {
    x = fabsf(x);
    if (ix < 0x3f980000u) {
      if (ix < 0x3f300000u) {
        id = 0;
        x = (2.0f * x - one) / (2.0f + x);
      } else {
        id = 1;
        x = (x - one) / (x + one);
      }
    } else {
      if (ix < 0x401c0000u) {
        id = 2;
        x = (x - 1.5f) / (one + 1.5f * x);
      } else {
        id = 3;
        x = -1.0f / x;
      }
    }
  }
  float z = x * x;
  const float w = z * z;
  const float s1 = z * (T0 + w * (T2 + w * (T4 + w * (T6 + w * (T8 + w * T10)))));
  const float s2 = w * (T1 + w * (T3 + w * (T5 + w * (T7 + w * T9))));
  if (id < 0) return x - x * (s1 + s2);
  const float hi = id == 0 ? hi0 : id == 1 ? hi1 : id == 2 ? hi2 : hi3;
  const float lo = id == 0 ? lo0 : id == 1 ? lo1 : id == 2 ? lo2 : lo3;
  z = hi - ((x * (s1 + s2) - lo) - x);
  return (hx & 0x80000000u) ? -z : z;
}

/// fdlibm atan2f. KLIM: the |y/x| exponent gap above which the quotient is not formed.
template <int KLIM>
WWB_HD float atan2f_t(float y, float x) {
  const float tiny = 1.0e-30f, pi_o_4 = asfloat(0x3f490fdbu), pi_o_2 = asfloat(0x3fc90fdbu),
              pi = asfloat(0x40490fdbu), pi_lo = asfloat(0xb3bbbd2eu);
  const int32_t hx = (int32_t)asuint(x), hy = (int32_t)asuint(y);
  const int32_t ix = hx & 0x7fffffff, iy = hy & 0x7fffffff;
  float z;
  if (ix > 0x7f800000 || iy > 0x7f800000) return x + y;
  if (hx == 0x3f800000) return atanf(y);
  const int m = ((hy >> 31) & 1) | ((hx >> 30) & 2);
  if (iy == 0) {
    switch (m) {
      case 0:
      case 1:
        return y;
      case 2:
        return pi + tiny;
      default:
        return -pi - tiny;
    }
  }
  if (ix == 0) return hy < 0 ? -pi_o_2 - tiny : pi_o_2 + tiny;
  if (ix == 0x7f800000) {
    if (iy == 0x7f800000) {
      switch (m) {
        case 0:
          return pi_o_4 + tiny;
        case 1:
          return -pi_o_4 - tiny;
        case 2:
          return 3.0f * pi_o_4 + tiny;
        default:
          return -3.0f * pi_o_4 - tiny;
      }
    }
    switch (m) {
      case 0:
        return 0.0f;
      case 1:
        return -0.0f;
      case 2:
        return pi + tiny;
      default:
        return -pi - tiny;
    }
  }
  if (iy == 0x7f800000) return hy < 0 ? -pi_o_2 - tiny : pi_o_2 + tiny;
  const int32_t k = (iy - ix) >> 23;
  if (k > KLIM) {
    z = pi_o_2 + 0.5f * pi_lo;
  } else if (hx < 0 && k < -KLIM) {
    z = 0.0f;
  } else {
    z = atanf(fabsf(y / x));
  }
  switch (m) {
    case 0:
      return z;
    case 1:
      return asfloat(asuint(z) ^ 0x80000000u);
    case 2:
      return pi - (z - pi_lo);
    default:
      return (z - pi_lo) - pi;
  }
}
#ifndef WWB_ATAN2F_KLIM
#define WWB_ATAN2F_KLIM 60
#endif
WWB_HC float atan2f(float y, float x) { return atan2f_t<WWB_ATAN2F_KLIM>(y, x); }

// ----------------------------------------------------------------------------------- log10f
/// fdlibm log10f over logf.
WWB_HC float log10f(float x) {
  const float two25 = asfloat(0x4c000000u), ivln10 = asfloat(0x3ede5bd9u),
              log10_2hi = asfloat(0x3e9a2080u), log10_2lo = asfloat(0x355427dbu);
  int32_t hx = (int32_t)asuint(x);
  int32_t k = 0;
  if (hx < 0x00800000) {
    if ((hx & 0x7fffffff) == 0) return -two25 / fabsf(x);
    if (hx < 0) return (x - x) / (x - x);
    k -= 25;
    x *= two25;
    hx = (int32_t)asuint(x);
  }
  if (hx >= 0x7f800000) return x + x;
  k += (hx >> 23) - 127;
  const int32_t i = (int32_t)(((uint32_t)k & 0x80000000u) >> 31);
  hx = (hx & 0x007fffff) | ((0x7f - i) << 23);
  const float y = (float)(k + i);
  x = asfloat((uint32_t)hx);
  const float z = y * log10_2lo + ivln10 * logf(x);
  return z + y * log10_2hi;
}

// --------------------------------------------------------------------------- double exp, tanh
// 2^(j/64), j = 0..63, as double-double (hi, lo): hi = 2^(j/64) rounded to double, lo the rounded
// remainder (generated; tests/test_libm.py regenerates and compares).
#define WWB_EXP2_64_TAB \
  {0x1.0000000000000p+0, 0x0.0p+0, 0x1.02c9a3e778061p+0, -0x1.19083535b085dp-56, \
   0x1.059b0d3158574p+0, 0x1.d73e2a475b465p-55, 0x1.0874518759bc8p+0, 0x1.186be4bb284ffp-57, \
   0x1.0b5586cf9890fp+0, 0x1.8a62e4adc610bp-54, 0x1.0e3ec32d3d1a2p+0, 0x1.03a1727c57b53p-59, \
   0x1.11301d0125b51p+0, -0x1.6c51039449b3ap-54, 0x1.1429aaea92de0p+0, -0x1.32fbf9af1369ep-54, \
   0x1.172b83c7d517bp+0, -0x1.19041b9d78a76p-55, 0x1.1a35beb6fcb75p+0, 0x1.e5b4c7b4968e4p-55, \
   0x1.1d4873168b9aap+0, 0x1.e016e00a2643cp-54, 0x1.2063b88628cd6p+0, 0x1.dc775814a8495p-55, \
   0x1.2387a6e756238p+0, 0x1.9b07eb6c70573p-54, 0x1.26b4565e27cddp+0, 0x1.2bd339940e9d9p-55, \
   0x1.29e9df51fdee1p+0, 0x1.612e8afad1255p-55, 0x1.2d285a6e4030bp+0, 0x1.0024754db41d5p-54, \
   0x1.306fe0a31b715p+0, 0x1.6f46ad23182e4p-55, 0x1.33c08b26416ffp+0, 0x1.32721843659a6p-54, \
   0x1.371a7373aa9cbp+0, -0x1.63aeabf42eae2p-54, 0x1.3a7db34e59ff7p+0, -0x1.5e436d661f5e3p-56, \
   0x1.3dea64c123422p+0, 0x1.ada0911f09ebcp-55, 0x1.4160a21f72e2ap+0, -0x1.ef3691c309278p-58, \
   0x1.44e086061892dp+0, 0x1.89b7a04ef80d0p-59, 0x1.486a2b5c13cd0p+0, 0x1.3c1a3b69062f0p-56, \
   0x1.4bfdad5362a27p+0, 0x1.d4397afec42e2p-56, 0x1.4f9b2769d2ca7p+0, -0x1.4b309d25957e3p-54, \
   0x1.5342b569d4f82p+0, -0x1.07abe1db13cadp-55, 0x1.56f4736b527dap+0, 0x1.9bb2c011d93adp-54, \
   0x1.5ab07dd485429p+0, 0x1.6324c054647adp-54, 0x1.5e76f15ad2148p+0, 0x1.ba6f93080e65ep-54, \
   0x1.6247eb03a5585p+0, -0x1.383c17e40b497p-54, 0x1.6623882552225p+0, -0x1.bb60987591c34p-54, \
   0x1.6a09e667f3bcdp+0, -0x1.bdd3413b26456p-54, 0x1.6dfb23c651a2fp+0, -0x1.bbe3a683c88abp-57, \
   0x1.71f75e8ec5f74p+0, -0x1.16e4786887a99p-55, 0x1.75feb564267c9p+0, -0x1.0245957316dd3p-54, \
   0x1.7a11473eb0187p+0, -0x1.41577ee04992fp-55, 0x1.7e2f336cf4e62p+0, 0x1.05d02ba15797ep-56, \
   0x1.82589994cce13p+0, -0x1.d4c1dd41532d8p-54, 0x1.868d99b4492edp+0, -0x1.fc6f89bd4f6bap-54, \
   0x1.8ace5422aa0dbp+0, 0x1.6e9f156864b27p-54, 0x1.8f1ae99157736p+0, 0x1.5cc13a2e3976cp-55, \
   0x1.93737b0cdc5e5p+0, -0x1.75fc781b57ebcp-57, 0x1.97d829fde4e50p+0, -0x1.d185b7c1b85d1p-54, \
   0x1.9c49182a3f090p+0, 0x1.c7c46b071f2bep-56, 0x1.a0c667b5de565p+0, -0x1.359495d1cd533p-54, \
   0x1.a5503b23e255dp+0, -0x1.d2f6edb8d41e1p-54, 0x1.a9e6b5579fdbfp+0, 0x1.0fac90ef7fd31p-54, \
   0x1.ae89f995ad3adp+0, 0x1.7a1cd345dcc81p-54, 0x1.b33a2b84f15fbp+0, -0x1.2805e3084d708p-57, \
   0x1.b7f76f2fb5e47p+0, -0x1.5584f7e54ac3bp-56, 0x1.bcc1e904bc1d2p+0, 0x1.23dd07a2d9e84p-55, \
   0x1.c199bdd85529cp+0, 0x1.11065895048ddp-55, 0x1.c67f12e57d14bp+0, 0x1.2884dff483cadp-54, \
   0x1.cb720dcef9069p+0, 0x1.503cbd1e949dbp-56, 0x1.d072d4a07897cp+0, -0x1.cbc3743797a9cp-54, \
   0x1.d5818dcfba487p+0, 0x1.2ed02d75b3707p-55, 0x1.da9e603db3285p+0, 0x1.c2300696db532p-54, \
   0x1.dfc97337b9b5fp+0, -0x1.1a5cd4f184b5cp-54, 0x1.e502ee78b3ff6p+0, 0x1.39e8980a9cc8fp-55, \
   0x1.ea4afa2a490dap+0, -0x1.e9c23179c2893p-54, 0x1.efa1bee615a27p+0, 0x1.dc7f486a4b6b0p-54, \
   0x1.f50765b6e4540p+0, 0x1.9d3e12dd8a18bp-54, 0x1.fa7c1819e90d8p+0, 0x1.74853f3a5931ep-55}
#if defined(__CUDACC__)
__device__ static const double kExp2_64Dev[128] = WWB_EXP2_64_TAB;
#endif
static const double kExp2_64Host[128] = WWB_EXP2_64_TAB;
WWB_HD double exp2_64(unsigned i) {
#if defined(__CUDA_ARCH__)
  return asdouble(tab_ld64(&kExp2_64Dev[i]));
#else
  return kExp2_64Host[i];
#endif
}

/// exp(x) in double: x = k ln2/64 + r, 2^(k/64) = 2^e 2^(j/64) from the double-double table,
/// e^r by a degree-11 Taylor sum (|r| <= ln2/128). Accurate to about 1 ulp; not glibc's bits
/// (W3SDB1 rounds the results it feeds to float).
WWB_HC double exp_d(double x) {
  if (x != x) return x + x;
  if (x > 709.78) return asdouble(0x7ff0000000000000ULL);
  if (x < -745.2) return 0.0;
  const double inv = 64.0 / 0.6931471805599453;
  const double kd = x * inv;
  const double kr = kd < 0 ? -(double)(int64_t)(-kd + 0.5) : (double)(int64_t)(kd + 0.5);
  const int64_t k = (int64_t)kr;
  // ln2/64 split hi + lo, hi with 33 significant bits so kr*hi is exact.
  const double ln2_64_hi = 0x1.62e42fefp-7, ln2_64_lo = 0x1.473de6af278edp-40;
  const double r = (x - kr * ln2_64_hi) - kr * ln2_64_lo;
  double p = 1.0 / 39916800.0;
  p = p * r + 1.0 / 3628800.0;
  p = p * r + 1.0 / 362880.0;
  p = p * r + 1.0 / 40320.0;
  p = p * r + 1.0 / 5040.0;
  p = p * r + 1.0 / 720.0;
  p = p * r + 1.0 / 120.0;
  p = p * r + 1.0 / 24.0;
  p = p * r + 1.0 / 6.0;
  p = p * r + 0.5;
  p = p * r * r + r;  // e^r - 1
  const int64_t j = ((k % 64) + 64) % 64;
  const int64_t e = (k - j) / 64;
  const double th = exp2_64(2 * (unsigned)j), tl = exp2_64(2 * (unsigned)j + 1);
  const double m = th + (th * p + (tl + tl * p));
  const int64_t e1 = e / 2, e2 = e - e1;
  return m * asdouble((uint64_t)(1023 + e1) << 52) * asdouble((uint64_t)(1023 + e2) << 52);
}

/// expm1(x) in double for |x| <= 1: the Taylor sum to x^19/19! (the first term left out is
/// below 2^-60 relative), without the cancellation of exp(x) - 1.
WWB_HD double expm1_small_d(double x) {
  double p = 1.0 / 121645100408832000.0;  // 1/19!
  const double inv[18] = {1.0 / 6402373705728000.0, 1.0 / 355687428096000.0,
                          1.0 / 20922789888000.0,   1.0 / 1307674368000.0,
                          1.0 / 87178291200.0,      1.0 / 6227020800.0,
                          1.0 / 479001600.0,        1.0 / 39916800.0,
                          1.0 / 3628800.0,          1.0 / 362880.0,
                          1.0 / 40320.0,            1.0 / 5040.0,
                          1.0 / 720.0,              1.0 / 120.0,
                          1.0 / 24.0,               1.0 / 6.0,
                          0.5,                      1.0};
  for (int i = 0; i < 18; ++i) p = p * x + inv[i];
  return p * x;
}

/// tanh(x) in double: expm1(2x) / (expm1(2x) + 2) for |x| < 0.5, 1 - 2 / (exp(2|x|) + 1) above.
WWB_HC double tanh_d(double x) {
  if (x != x) return x + x;
  const double ax = x < 0 ? -x : x;
  if (ax > 22.0) return x < 0 ? -1.0 : 1.0;
  if (ax < 0x1p-28) return x;
  double t;
  if (ax < 0.5) {
    const double em1 = expm1_small_d(2.0 * ax);
    t = em1 / (em1 + 2.0);
  } else {
    const double e2 = exp_d(2.0 * ax);
    t = 1.0 - 2.0 / (e2 + 1.0);
  }
  return x < 0 ? -t : t;
}

}  // namespace dm
}  // namespace wwb
