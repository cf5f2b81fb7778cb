/* oracle/mvec_scalar.c -- TEST INFRASTRUCTURE ONLY.
 *
 * The two glibc libmvec entry points the reference's ST4 calls explicitly
 * (kokkos/src/ww_kokkos/st4_libmvec.hpp:25-27: _ZGVbN4vv_powf, _ZGVbN4v_expf, SSE 4-lane),
 * defined here as four scalar glibc powf/expf calls, one per lane, with hidden visibility so
 * that the reference objects of libref_ww3_scalar.so bind to them inside the library. The
 * reference then computes, at those five loops (w3src4md.F90:316, :317, :2315, :2500, :2509),
 * what any implementation without libmvec computes: scalar glibc powf and expf in every lane.
 */
#include <math.h>
#include <xmmintrin.h>

__attribute__((visibility("hidden"))) __m128 _ZGVbN4vv_powf(__m128 x, __m128 y) {
  float a[4], b[4], r[4];
  _mm_storeu_ps(a, x);
  _mm_storeu_ps(b, y);
  for (int l = 0; l < 4; ++l) r[l] = powf(a[l], b[l]);
  return _mm_loadu_ps(r);
}

__attribute__((visibility("hidden"))) __m128 _ZGVbN4v_expf(__m128 x) {
  float a[4], r[4];
  _mm_storeu_ps(a, x);
  for (int l = 0; l < 4; ++l) r[l] = expf(a[l]);
  return _mm_loadu_ps(r);
}

/* The two libmvec entry points of the reference's W3OUTG (iogo_w3outg.hpp:37-40: the THMP
 * sine and cosine of the space-time extremes), likewise scalar per lane. */
__attribute__((visibility("hidden"))) __m128 _ZGVbN4v_sinf(__m128 x) {
  float a[4], r[4];
  _mm_storeu_ps(a, x);
  for (int l = 0; l < 4; ++l) r[l] = sinf(a[l]);
  return _mm_loadu_ps(r);
}

__attribute__((visibility("hidden"))) __m128 _ZGVbN4v_cosf(__m128 x) {
  float a[4], r[4];
  _mm_storeu_ps(a, x);
  for (int l = 0; l < 4; ++l) r[l] = cosf(a[l]);
  return _mm_loadu_ps(r);
}
