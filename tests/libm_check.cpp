// tests/libm_check.cpp -- compares the host build of ww3-gpu_b200/csrc/libm_dev.cuh with this
// host's glibc. Usage: libm_check <function> <stride>; checks every stride-th float bit pattern
// (stride 1 = all 2^32) for unary functions, and stride-thinned seeded pairs for powf, atan2f,
// and prints the number of mismatching inputs per variant ("variant v n").
#include <omp.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../ww3-gpu_b200/csrc/libm_dev.cuh"

using namespace wwb::dm;

static inline bool same(float a, float b) {
  return asuint(a) == asuint(b) || (std::isnan(a) && std::isnan(b));
}
static inline uint64_t mix(long long i) {
  uint64_t h = static_cast<uint64_t>(i) * 0x9E3779B97F4A7C15ULL;
  h ^= h >> 29;
  h *= 0xBF58476D1CE4E5B9ULL;
  h ^= h >> 32;
  return h;
}

int main(int argc, char** argv) {
  const char* fn = argc > 1 ? argv[1] : "expf";
  const long long stride = argc > 2 ? std::atoll(argv[2]) : 1;
  long long bad[8] = {0}, n = 0;
  const bool unary = std::strcmp(fn, "powf") != 0 && std::strcmp(fn, "atan2f") != 0;
  if (unary) {
#pragma omp parallel for schedule(static) reduction(+ : bad[:8], n)
    for (long long u = 0; u < (1LL << 32); u += stride) {
      const float x = asfloat(static_cast<uint32_t>(u));
      ++n;
      if (!std::strcmp(fn, "expf")) {
        const float g = ::expf(x);
#define C(V) if (!same(expf_t<V>(x), g)) ++bad[V];
        C(0) C(1) C(2) C(3) C(4) C(5) C(6) C(7)
#undef C
      } else if (!std::strcmp(fn, "logf")) {
        if (!same(wwb::dm::logf(x), ::logf(x))) ++bad[0];
      } else if (!std::strcmp(fn, "sincosf")) {
        float gs, gc, s, c;
        ::sincosf(x, &gs, &gc);
        wwb::dm::sincosf(x, &s, &c);
        if (!same(s, gs) || !same(c, gc)) ++bad[0];
        if (!same(s, ::sinf(x)) || !same(c, ::cosf(x))) ++bad[1];
      } else if (!std::strcmp(fn, "tanhf")) {
        if (!same(wwb::dm::tanhf(x), ::tanhf(x))) ++bad[0];
      } else if (!std::strcmp(fn, "sinhf")) {
        if (!same(wwb::dm::sinhf(x), ::sinhf(x))) ++bad[0];
      } else if (!std::strcmp(fn, "coshf")) {
        if (!same(wwb::dm::coshf(x), ::coshf(x))) ++bad[0];
      } else if (!std::strcmp(fn, "atanf")) {
        if (!same(wwb::dm::atanf(x), ::atanf(x))) ++bad[0];
      } else if (!std::strcmp(fn, "log10f")) {
        if (!same(wwb::dm::log10f(x), ::log10f(x))) ++bad[0];
      }
    }
  } else {
#pragma omp parallel for schedule(static) reduction(+ : bad[:8], n)
    for (long long i = 0; i < (1LL << 32) / stride; ++i) {
      const uint64_t h = mix(i);
      float x = asfloat(static_cast<uint32_t>(h)), y = asfloat(static_cast<uint32_t>(h >> 32));
      ++n;
      if (!std::strcmp(fn, "powf")) {
        if (i & 1) {  // positive bases, exponents in [0.25, 0.5) and small multiples of 1/4
          x = std::fabs(x);
          y = asfloat(0x3e800000u + (static_cast<uint32_t>(h >> 40) & 0x7ffff));
        }
        if ((i & 3) == 2) y = static_cast<float>(static_cast<int>((h >> 50) % 16) - 8) * 0.25f;
        if (!same(wwb::dm::powf(x, y), ::powf(x, y))) ++bad[0];
      } else {
        if (i & 1) {  // arguments of moderate size, as the stress directions have
          x = static_cast<float>(static_cast<int>(h % 2001) - 1000) * 0.013f;
          y = static_cast<float>(static_cast<int>((h >> 20) % 2001) - 1000) * 0.007f;
        }
        if (!same(wwb::dm::atan2f(y, x), ::atan2f(y, x))) ++bad[0];
      }
    }
  }
  std::printf("checked %lld\n", n);
  for (int v = 0; v < 8; ++v) std::printf("variant %d %lld\n", v, bad[v]);
  std::printf("default %d\n", std::strcmp(fn, "expf") ? 0 : WWB_EXPF_FUSE);
  return 0;
}
