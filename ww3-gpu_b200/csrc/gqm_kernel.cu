// ww3-gpu_b200/csrc/gqm_kernel.cu
// The table builders of the GQM form of NL1 (INSNLGQM's helpers): COUPLE, the Webb four-wave
// coupling coefficient, batched on the device in FP64 (one thread per wavenumber quadruplet);
// GAULEG (Gauss-Legendre abscissas and weights) and F1F1F1 (the f1/f ratio layouts) on the
// host, where the reference runs them too (they call the host's double cos and pow, whose bits
// the device does not reproduce). The C ABI is ww_snl1_gqm_couple, ww_snl1_gqm_gauleg and
// ww_snl1_gqm_f1f1f1 (include/ww_b200.h).
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/snl1_couple.hpp:37-88 (COUPLE), snl1_gauleg.hpp:28-61
// (GAULEG), snl1_f1f1f1.hpp:37-145 (F1F1F1); WW3 w3snl1md.F90:1185-1500. The reference exports
// no C entry for them (its W3SRCE leaves IQTYPE <= 0 to the Fortran).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <exception>

#include "wwb_common.hpp"

namespace wwb {
namespace {

Status g_gqm_status;

// COEF = PI*GRAV*GRAV/4.D0 with PI = ACOS(-1.) of default kind (the float nearest pi, widened)
// and GRAV the REAL 9.806, as gfortran folds it; ZERO = 1.D-10 (w3snl1md.F90:1242-1244).
constexpr double kPiF = static_cast<double>(static_cast<float>(3.14159265358979323846));
constexpr double kGravF = static_cast<double>(9.806f);
constexpr double kCoef = kPiF * kGravF * kGravF / 4.0;
constexpr double kZero = 1.e-10;

/// COUPLE (w3snl1md.F90:1185-1307) for one quadruplet: returns the coefficient, sets diag to the
/// bits of the Fortran's warnings (1: term 1-3 is 0/0, 2: term 1-3 infinite, 4 and 8 the same for
/// term 1-4; such a term is left out). Every expression in the Fortran's association order.
__device__ double couple(double xk1, double yk1, double xk2, double yk2, double xk3, double yk3,
                         double xk4, double yk4, int& diag) {
  diag = 0;
  const double rk1 = sqrt(xk1 * xk1 + yk1 * yk1);
  const double rk2 = sqrt(xk2 * xk2 + yk2 * yk2);
  const double rk3 = sqrt(xk3 * xk3 + yk3 * yk3);
  const double rk4 = sqrt(xk4 * xk4 + yk4 * yk4);
  const double wk1 = sqrt(rk1), wk2 = sqrt(rk2), wk3 = sqrt(rk3), wk4 = sqrt(rk4);
  const double s12 = xk1 * xk2 + yk1 * yk2;
  const double s13 = xk1 * xk3 + yk1 * yk3;
  const double s14 = xk1 * xk4 + yk1 * yk4;
  const double s23 = xk2 * xk3 + yk2 * yk3;
  const double s24 = xk2 * xk4 + yk2 * yk4;
  const double s34 = xk3 * xk4 + yk3 * yk4;
  const double w1p2 = sqrt((xk1 + xk2) * (xk1 + xk2) + (yk1 + yk2) * (yk1 + yk2));
  const double w1m3 = sqrt((xk1 - xk3) * (xk1 - xk3) + (yk1 - yk3) * (yk1 - yk3));
  const double w1m4 = sqrt((xk1 - xk4) * (xk1 - xk4) + (yk1 - yk4) * (yk1 - yk4));
  const double q12 = (wk1 + wk2) * (wk1 + wk2);
  const double q13 = (wk1 - wk3) * (wk1 - wk3);
  const double q14 = (wk1 - wk4) * (wk1 - wk4);
  double ddd = 2.00 * q12 * (rk1 * rk2 - s12) * (rk3 * rk4 - s34) / (w1p2 - q12) +
               0.50 * (s12 * s34 + s13 * s24 + s14 * s23) +
               0.25 * (s13 + s24) * q13 * q13 -
               0.25 * (s12 + s34) * q12 * q12 +
               0.25 * (s14 + s23) * q14 * q14 +
               2.50 * rk1 * rk2 * rk3 * rk4 +
               q12 * q13 * q14 * (rk1 + rk2 + rk3 + rk4);
  const double deno13 = w1m3 - q13;
  const double nume13 = 2.00 * q13 * (rk1 * rk3 + s13) * (rk2 * rk4 + s24);
  if (fabs(deno13) < kZero)
    diag |= fabs(nume13) < kZero ? 1 : 2;
  else
    ddd = ddd + nume13 / deno13;
  const double deno14 = w1m4 - q14;
  const double nume14 = 2.00 * q14 * (rk1 * rk4 + s14) * (rk2 * rk3 + s23);
  if (fabs(deno14) < kZero)
    diag |= fabs(nume14) < kZero ? 4 : 8;
  else
    ddd = ddd + nume14 / deno14;
  return kCoef * ddd * ddd / (wk1 * wk2 * wk3 * wk4);
}

/// k: (8, n) column-major, the quadruplet (XK1, YK1, XK2, YK2, XK3, YK3, XK4, YK4) per column.
__global__ void couple_kernel(int n, const double* __restrict__ k, double* __restrict__ out,
                              int* __restrict__ diag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* c = k + static_cast<size_t>(i) * 8;
  int d = 0;
  out[i] = couple(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], d);
  if (diag) diag[i] = d;
}

}  // namespace
}  // namespace wwb

using namespace wwb;

extern "C" {

int ww_snl1_gqm_couple(int n, const double* k, double* coef, int* diag) {
  try {
    if (!runtime().ready)
      return g_gqm_status.fail(WW_KOKKOS_ERR_NOT_INITIALISED, "ww_snl1_gqm_couple before init");
    if (n < 0 || (n > 0 && (!k || !coef)))
      return g_gqm_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_gqm_couple: bad size or null");
    if (n == 0) {
      g_gqm_status.ok();
      return WW_KOKKOS_OK;
    }
    cudaStream_t s = runtime().stream;
    double *dk = nullptr, *dc = nullptr;
    int* dd = nullptr;
    struct Free {
      void* p[3];
      ~Free() {
        for (void* q : p)
          if (q) cudaFree(q);
      }
    } fr{{nullptr, nullptr, nullptr}};
    WWB_CHECK(cudaMalloc(&dk, sizeof(double) * 8 * static_cast<size_t>(n)));
    fr.p[0] = dk;
    WWB_CHECK(cudaMalloc(&dc, sizeof(double) * static_cast<size_t>(n)));
    fr.p[1] = dc;
    if (diag) {
      WWB_CHECK(cudaMalloc(&dd, sizeof(int) * static_cast<size_t>(n)));
      fr.p[2] = dd;
    }
    WWB_CHECK(cudaMemcpyAsync(dk, k, sizeof(double) * 8 * static_cast<size_t>(n),
                              cudaMemcpyHostToDevice, s));
    couple_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, dk, dc, dd);
    WWB_CHECK(cudaGetLastError());
    WWB_CHECK(cudaMemcpyAsync(coef, dc, sizeof(double) * static_cast<size_t>(n),
                              cudaMemcpyDeviceToHost, s));
    if (diag)
      WWB_CHECK(cudaMemcpyAsync(diag, dd, sizeof(int) * static_cast<size_t>(n),
                                cudaMemcpyDeviceToHost, s));
    WWB_CHECK(cudaStreamSynchronize(s));
    g_gqm_status.ok();
    return WW_KOKKOS_OK;
  } catch (const std::exception& e) {
    return g_gqm_status.fail(WW_KOKKOS_ERR_KERNEL, e.what());
  }
}

int ww_snl1_gqm_gauleg(int npoin, double* w_leg, double* x_leg) {
  if (npoin < 1) return WW_KOKKOS_OK;  // the Fortran's loop writes nothing
  if (!w_leg || !x_leg)
    return g_gqm_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_gqm_gauleg: null array");
  // GAULEG (w3snl1md.F90:1310-1346): per root, Newton steps on P_NPOIN from the Tricomi guess
  // cos(pi (i - 1/4) / (NPOIN + 1/2)) with PI = ACOS(-1.) of default kind, until a step is at
  // most EPS = 3.D-14. The Fortran's loop has no limit; here 1000 steps without convergence is
  // a failure (KERNEL), which no NPOIN the Fortran can finish reaches.
  const double pi = kPiF, eps = 3.e-14;
  const int m = (npoin + 1) / 2;
  for (int i = 1; i <= m; ++i) {
    double z = std::cos(pi * (static_cast<double>(i) - 0.25) / (static_cast<double>(npoin) + 0.5));
    double p1 = 1.0, p2 = 0.0, pp = 0.0;
    int it = 0;
    for (;; ++it) {
      if (it == 1000)
        return g_gqm_status.fail(WW_KOKKOS_ERR_KERNEL, "ww_snl1_gqm_gauleg: Newton did not converge");
      p1 = 1.0;
      p2 = 0.0;
      for (int j = 1; j <= npoin; ++j) {
        const double p3 = p2;
        p2 = p1;
        const double dj = static_cast<double>(j);
        p1 = ((2.0 * dj - 1.0) * z * p2 - (dj - 1.0) * p3) / dj;
      }
      pp = static_cast<double>(npoin) * (z * p1 - p2) / (z * z - 1.0);
      const double z1 = z;
      z = z - p1 / pp;
      if (std::fabs(z - z1) <= eps) break;
    }
    x_leg[i - 1] = -z;
    x_leg[npoin - i] = z;
    w_leg[i - 1] = 2.0 / ((1.0 - z * z) * (pp * pp));
    w_leg[npoin - i] = w_leg[i - 1];
  }
  g_gqm_status.ok();
  return WW_KOKKOS_OK;
}

int ww_snl1_gqm_f1f1f1(int* nf1, int iq_om1, double* f1sf) {
  if (!nf1 || !f1sf) return -g_gqm_status.fail(WW_KOKKOS_ERR_BAD_SHAPE, "ww_snl1_gqm_f1f1f1: null");
  // F1F1F1 (w3snl1md.F90:1349-1500): the ratios f1/f for layout IQ_OM1. 1, 2, 3, 7: fixed lists
  // (15, 27, 12, 21 entries) that expect NF1 = 14, 26, 11, 20; 4: 41 geometric entries around
  // 1/3 with ratio 9**(1/20), NF1 set to 40; 5: NF1+1 geometric entries from 1/3 with ratio
  // 9**(1/NF1); 6: NF1+1 arithmetic entries from 1/3 in steps of (3 - 1/3)/NF1. Returns 0, or
  // the bit of the message the Fortran writes when NF1 does not fit the layout (1, 2, 4, 8, 16
  // for layouts 1, 2, 3, 4, 7).
  static const double kL1[] = {0.30, 0.40, 0.50, 0.60, 0.70, 0.80, 0.90, 1.00,
                               1.11, 1.25, 1.42, 1.67, 2.00, 2.50, 3.30};
  static const double kL2[] = {0.32, 0.35, 0.39, 0.44, 0.50, 0.56, 0.63, 0.70, 0.78,
                               0.86, 0.92, 0.97, 1.00, 1.03, 1.08, 1.13, 1.20, 1.28,
                               1.37, 1.48, 1.50, 1.65, 1.85, 2.10, 2.40, 2.70, 3.20};
  static const double kL3[] = {0.30, 0.48, 0.64, 0.78, 0.90, 1.00,
                               1.12, 1.28, 1.50, 1.80, 2.40, 3.40};
  static const double kL7[] = {1.0 / 3.0, 0.40, 0.46, 0.52, 0.60, 0.70, 0.79,
                               0.86,      0.92, 0.97, 1.00, 1.04, 1.10, 1.18,
                               1.28,      1.42, 1.60, 1.84, 2.14, 2.52, 3.00};
  auto copy = [&](const double* t, int len) {
    for (int i = 0; i < len; ++i) f1sf[i] = t[i];
  };
  int diag = 0;
  switch (iq_om1) {
    case 1:
      if (*nf1 != 14) diag = 1;
      copy(kL1, 15);
      break;
    case 2:
      if (*nf1 != 26) diag = 2;
      copy(kL2, 27);
      break;
    case 3:
      if (*nf1 != 11) diag = 4;
      copy(kL3, 12);
      break;
    case 4: {
      if (*nf1 != 40) diag = 8;
      // 9**(1/20) correctly rounded (gfortran folds the power at compile time):
      // 1.1161231740339044, 0x1.1dba3f92c888bp+0.
      const double raison = 0x1.1dba3f92c888bp+0;
      const int mm = 10;
      *nf1 = 2 * mm + 20;
      f1sf[mm] = 1.0 / 3.0;
      for (int i = mm + 2; i <= *nf1 + 1; ++i) f1sf[i - 1] = f1sf[i - 2] * raison;
      for (int i = mm; i >= 1; --i) f1sf[i - 1] = f1sf[i] / raison;
      break;
    }
    case 5: {
      const double raison = std::pow(9.0, 1.0 / static_cast<double>(*nf1));
      f1sf[0] = 1.0 / 3.0;
      for (int i = 2; i <= *nf1 + 1; ++i) f1sf[i - 1] = f1sf[i - 2] * raison;
      break;
    }
    case 6: {
      const double step = (3.0 - 1.0 / 3.0) / static_cast<double>(*nf1);
      f1sf[0] = 1.0 / 3.0;
      for (int i = 2; i <= *nf1 + 1; ++i) f1sf[i - 1] = f1sf[i - 2] + step;
      break;
    }
    case 7:
      if (*nf1 != 20) diag = 16;
      copy(kL7, 21);
      break;
    default:
      break;
  }
  g_gqm_status.ok();
  return diag;
}

int ww_snl1_gqm_last_error(void) { return g_gqm_status.get(); }

}  // extern "C"
