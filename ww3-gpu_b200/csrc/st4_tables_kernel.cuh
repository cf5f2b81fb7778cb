// ww3-gpu_b200/csrc/st4_tables_kernel.cuh
// INSIN4, the ST4 initialisation, on the device (st4_tables_kernel.cu): the saturation indices
// and weights, IKTAB, DCKI and QBI of the bandwidth-integrated breaking, the cumulative weights
// CUMULW and, when FLTABS, the stress tables TAUT (TABU_STRESS), TAUHFT (TABU_TAUHF) and TAUHFT2
// (TABU_TAUHF2), bit for bit as the reference's host code builds them.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/st4_insin4.cpp:96-264, st4_tabu_stress.cpp:20-73,
// st4_tabu_tauhf.cpp:18-76, st4_tabu_tauhf2.cpp:25-101 (w3src4md.F90:1014-1831); the shapes of
// st4_arrays.hpp:117-132.
#pragma once

#include <cuda_runtime.h>

#include "st4_params.hpp"

namespace wwb {

/// The arrays INSIN4 reads, on the device: SIG, DSIP (0:MK+1), TH (MTH), ECOS (MSPEC+MTH).
struct St4TablesIn {
  const float *sig, *dsip, *th, *ecos;
};

/// INSIN4's outputs on the device, column-major with the reference's shapes; a null pointer is a
/// table not built. SATWEIGHTS, SATINDICES (2*(MTH/2-1)+1, MTH); IKTAB (MK, NDTAB); DCKI, QBI
/// (NKHS, NKD); CUMULW (MSPEC, MSPEC); TAUT (0:ITAUMAX, 0:JUMAX); TAUHFT (0:IUSTAR, 0:IALPHA);
/// TAUHFT2 (0:IUSTAR, 0:IALPHA, 0:ILEVTAIL).
struct St4TablesOut {
  float* satweights;
  int* satindices;
  int* iktab;
  float *dcki, *qbi, *cumulw, *taut, *tauhft, *tauhft2;
};

/// The branches INSIN4 takes and the W3SRC4MD module scalars it sets, from the packet alone.
struct St4TablesPlan {
  bool taut, tauhf, tauhf2;  // TABU_STRESS, TABU_TAUHF (its TAUHFT kept), TABU_TAUHF2
  bool sat, bck, cumul;      // SSDSDTH < 180, SSDSBCK > 0, SSDSC(3) < 0
  int nsat, sdsnth, dikcumul;
  float delust, delalp, deltauw, delu, deltail;  // the packet's values where INSIN4 sets none
};
St4TablesPlan st4_tables_plan(const st4::Params& p, bool fltabs);

/// Builds every table of `plan` into `out` on stream s (TAUHFT2, a long serial recurrence per
/// entry, on stream s2, joined back into s before the call returns to the host's order).
void launch_st4_tables(const st4::Params& p, const St4TablesPlan& plan, const St4TablesIn& in,
                       const St4TablesOut& out, cudaStream_t s, cudaStream_t s2);

}  // namespace wwb
