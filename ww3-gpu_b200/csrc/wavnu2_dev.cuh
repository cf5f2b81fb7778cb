// ww3-gpu_b200/csrc/wavnu2_dev.cuh
// WAVNU2 on the device, shared by DISTAB (wave_kernel.cu) and INSIN4's IKTAB
// (st4_tables_kernel.cu). Both reference call sites compile the same statements (ww3-gpu
// kokkos/src/ww_kokkos/disp_distab.hpp:77-130 and st4_insin4.cpp:38-90, w3dispmd.F90:204-346);
// their operand orders differ only by commuted products (kGrav*h for h*kGrav, 2*k for k+k), which
// round the same.
#pragma once

#include "libm_dev.cuh"

namespace wwb {
namespace disp {

constexpr float kGravD = 9.806f;  // CONSTANTS GRAV

/// WAVNU2(W, H, K, CG, EPS, NMAX, ICON) (w3dispmd.F90:204-346): Newton iteration on
/// w**2 = g k tanh(k h); ICON is not returned (neither caller reads it).
__device__ __forceinline__ void wavnu2(float w, float h, float& k, float& cg, float eps,
                                       int nmax) {
  const float zero = 0.0f;
  float kold = zero;
  const float w0 = fabsf(w);
  if (sqrtf(kGravD / h) > w0) {
    k = w0 / sqrtf(h * kGravD);
  } else {
    k = w * w / kGravD;
  }
  for (int i = 1; i <= nmax; ++i) {
    const float dif = fabsf(k - kold);
    const float rdif = (k != zero) ? dif / k : zero;
    if (dif < eps && rdif < eps) break;
    kold = k;
    const float gk = kold * kGravD;
    const float kh = h * kold;
    const float th = dm::tanhf(kh);
    const float f = gk * th - w * w;
    float fd;
    if (kh > 25.0f) {
      fd = th * kGravD;
    } else {
      const float c = dm::coshf(kh);
      fd = th * kGravD + (h * gk) / (c * c);
    }
    k = kold - f / fd;
  }
  const float kh2 = h * (k + k);
  const float cgd = w0 / k * 0.5f;
  cg = (kh2 > 25.0f) ? cgd : cgd * (1.0f + kh2 / dm::sinhf(kh2));
  if (w < zero) {
    k = -k;
    cg = -cg;
  }
}

}  // namespace disp
}  // namespace wwb
