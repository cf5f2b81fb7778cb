// ww3-gpu_b200/csrc/snl1_kernel.cuh
// W3SNL1 (the DIA) on B200: kernel parameters and launchers.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/snl1_team.hpp:351-497 (WW3 w3snl1md.F90 W3SNL1,
// lines 115-473) and its batch launch snl1_dia.cpp:30-69.
#pragma once

#include <cuda_runtime.h>

namespace wwb {

/// Everything the DIA kernels read besides the batch, passed by value as a kernel parameter.
struct Snl1Dev {
  int nk, nth, nfr, nfrhgh, nfrchg, nspec, nspecx;
  float dal1, dal2, dal3;
  float awg[8], swg[8];
  float snlc1, kdcon, kdmn, snls1, snls2, snls3, fachfe;
  int shift[8];             ///< row-shift form: IT_n(ITH) - ITH
  int ifrp, ifrm;           ///< row-shift form: IF1 = IFR + IFRP, IF3 = MAX(0, IFR + IFRM)
  const int* ifrow;         ///< device, 8 x NFRCHG (row-shift form)
  const float* af11_row;    ///< device, NFRCHG (row-shift form)
  const int* ipim;          ///< device, 16 x NSPECX (gather form)
  const int* ic;            ///< device, 16 x NSPEC (gather form)
  const float* af11;        ///< device, NSPECX (gather form)
  const float* sig;         ///< device, NK
  /// Test of the failure path (0 in every normal run): bytes added to the bytes each CTA of the
  /// pair kernels expects for its first bulk copy, which therefore never completes, so its
  /// bounded wait runs out and the launch reports it (ww_snl1_test_stall).
  int stall_tx;
};

enum Snl1Kernel {
  kSnl1Auto = 0,
  kSnl1Gather = 1,
  kSnl1RowShift = 2,
  kSnl1Band = 3,
  kSnl1Tile = 4,
  kSnl1Pair = 5,  ///< the band kernel over two points at once (paired FP32 additions)
  kSnl1PairGeneral = 6,  ///< the pair kernel's general form even where its 36-direction tile fits
};

/// Dynamic shared memory of each kernel, bytes.
size_t snl1_gather_smem(const Snl1Dev& p);
size_t snl1_rowshift_smem(const Snl1Dev& p);
size_t snl1_band_smem(const Snl1Dev& p);

/// Whether the band kernel can run these tables (row-shift form, NTH within one CTA, the
/// rows of a band within its register windows).
bool snl1_band_ok(const Snl1Dev& p);

size_t snl1_pair_smem(const Snl1Dev& p);

/// Whether the pair kernel can run these tables (the band kernel's conditions, interaction
/// arrays of at most 1536 bins, NSPEC and NK multiples of 4 for its bulk copies).
bool snl1_pair_ok(const Snl1Dev& p);

/// Whether a compile-time tile instance of the band kernel fits these tables (NTH 36 or 24,
/// NSPEC and NK multiples of 4 for the bulk copies).
bool snl1_tile_ok(const Snl1Dev& p);

/// Device status word of the band kernel's bounded waits: nonzero after a wait gave up.
int snl1_take_error();

/// Launch W3SNL1 on npts points; a, s, d (nspec, npts) and cg (nk, npts) column-major,
/// kdmean (npts), all device pointers. Throws CudaError on a launch failure.
void launch_snl1(int kernel, const Snl1Dev& p, int npts, const float* a, const float* cg,
                 const float* kdmean, float* s, float* d, cudaStream_t stream);

/// The device array behind ww_snl1_noalloc on the current device: `floats` floats at `base`
/// (256-byte aligned) and an int error flag. The first call on a device resolves the addresses
/// (cudaGetSymbolAddress); later calls return them.
struct Snl1StaticScratch {
  float* base = nullptr;
  size_t floats = 0;
  int* err = nullptr;
};
Snl1StaticScratch snl1_static_scratch();

/// launch_snl1 with the band and tile kernels' bulk-copy failures reported in `err` (non-null,
/// zero before the launch) instead of the shared flag that snl1_take_error reads.
void launch_snl1_err(int kernel, const Snl1Dev& p, int npts, const float* a, const float* cg,
                     const float* kdmean, float* s, float* d, int* err, cudaStream_t stream);

/// The pair kernel (the band kernel where the pair kernel does not fit, or the arrays are not
/// 16-byte aligned) on the points pidx[0 .. min(capacity, *pcount)) of the arrays (pidx and
/// pcount device pointers; the count may be written by an earlier kernel on `stream`). Returns
/// false, launching nothing, when the band kernel cannot run these tables.
bool launch_snl1_list(const Snl1Dev& p, int capacity, const int* pidx, const int* pcount,
                      const float* a, const float* cg, const float* kdmean, float* s, float* d,
                      int* err, cudaStream_t stream);

}  // namespace wwb
