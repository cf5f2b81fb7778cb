// ww3-gpu_b200/csrc/utrn_kernel.cuh
// W3UTRN on the device (utrn_kernel.cu): ATRNX/ATRNY of the PR3 propagation.
// Reference: ww3-gpu kokkos/src/ww_kokkos/updt_utrn.hpp:93-362.
#pragma once

#include <cuda_runtime.h>

namespace wwb {

/// W3UTRN's scalars (updt_utrn.hpp:93-104). trny_before is the REAL in memory just before
/// TRNY(1), which the Fortran reads as TRNY(0) when cell 1 is a sea point under TRFLAG 1, 3, 5.
struct UtrnGrid {
  int nx, ny, nsea, trflag;
  float fice0, ficen, ficel, ffacberg;
  int flagll;
  float trny_before;
};

/// Whether the ice passes run (TRFLAG >= 3 and FICEN - FICE0 >= 1.E-6, as W3UTRN tests it):
/// then trix, triy (NY*NX each) are the work of launch_utrn.
bool utrn_needs_ice(const UtrnGrid& g);

/// W3UTRN on device arrays: mapsf (NSEA,3), mapsta, hpfac, hqfac (NY,NX), trnx, trny (NY*NX),
/// ice (0:NSEA), berg (NSEA) in; atrnx, atrny (NY*NX, -1:1) out.
void launch_utrn(const UtrnGrid& g, const int* mapsf, const int* mapsta, const float* trnx,
                 const float* trny, const float* hpfac, const float* hqfac, const float* ice,
                 const float* berg, float* atrnx, float* atrny, float* trix, float* triy,
                 cudaStream_t s);

}  // namespace wwb
