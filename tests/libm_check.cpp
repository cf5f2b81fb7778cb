// tests/libm_check.cpp -- compares the host build of ww3-gpu_b200/csrc/libm_dev.cuh's expf with
// this host's glibc expf. Usage: libm_check <stride> [variant]; checks every stride-th float bit
// pattern (stride 1 = all 2^32) and prints the number of mismatching inputs per variant.
#include <omp.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "../ww3-gpu_b200/csrc/libm_dev.cuh"

int main(int argc, char** argv) {
  const long long stride = argc > 1 ? std::atoll(argv[1]) : 1;
  long long bad[8] = {0};
  long long n = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad[:8], n)
  for (long long u = 0; u < (1LL << 32); u += stride) {
    const float x = wwb::dm::asfloat(static_cast<uint32_t>(u));
    const float g = ::expf(x);
    const uint32_t gb = wwb::dm::asuint(g);
    ++n;
#define CHK(V)                                                         \
  {                                                                    \
    const float m = wwb::dm::expf_t<V>(x);                             \
    if (wwb::dm::asuint(m) != gb && !(std::isnan(m) && std::isnan(g))) \
      ++bad[V];                                                        \
  }
    CHK(0) CHK(1) CHK(2) CHK(3) CHK(4) CHK(5) CHK(6) CHK(7)
#undef CHK
  }
  std::printf("checked %lld\n", n);
  for (int v = 0; v < 8; ++v) std::printf("variant %d %lld\n", v, bad[v]);
  std::printf("default %d\n", WWB_EXPF_FUSE);
  return 0;
}
