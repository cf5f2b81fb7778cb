// ww3-gpu_b200/csrc/wave_kernel.cuh
// W3WAVE's per-step support routines on the device (wave_kernel.cu): W3GATH and W3SCAT (one
// spectral component between VA and a 2-D field), W3UWND (the wind at the model time), W3DZXY
// (gradients of a sea-point field), DISTAB (the dispersion tables) and W3CFLXY (the largest
// spatial CFL number of each sea point).
// Reference: ww3-gpu kokkos/src/ww_kokkos/wave_gath_scat.hpp, updt_uwnd.hpp, updt_dzxy.hpp,
// disp_distab.hpp, prop_cflxy.hpp; the C ABI of the first four in
// kokkos/src/fortran_iface/wave_support_shim.cpp (W3CFLXY is called from the device W3WAVE
// driver only, wave_w3wave.hpp:548-574).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace wwb {

/// W3GATH: FIELD(1-NY:NY*(NX+2)) (nf = NY*(NX+3) floats) zeroed, then FIELD(IXY) = row[ISEA]
/// for ISEA = 1..nsea, IXY = ixy[ISEA-1] (MAPSF(:,3)); row is VA(ISPEC, 0:NSEA).
void launch_wave_gath(int nsea, int ny, size_t nf, const float* row, const int* ixy,
                      float* field, cudaStream_t s);

/// W3SCAT: row[ISEA] = FIELD(IXY) where MAPSTA(IXY) /= 0, ISEA = 1..nsea.
void launch_wave_scat(int nsea, int ny, const int* mapsta, const float* field, const int* ixy,
                      float* row, cudaStream_t s);

/// W3UWND's arrays on the device: mapsf (MSEA,3); the six input fields (NX,NY); the NSEA arrays.
struct UwndArgs {
  int nsea, msea, nx, ny;
  bool flfrst, flcur;
  float rd, rwindc;
  const int* mapsf;
  const float *wx0, *wy0, *dt0, *wxn, *wyn, *dtn, *cx, *cy;
  float *ua0, *uai, *ud0, *udi, *as0, *asi, *ua, *ud, *as, *u10, *u10d;
};
void launch_wave_uwnd(const UwndArgs& a, cudaStream_t s);

/// W3DZXY on the device: zz (NSEA), mapsta, mapfs, dpdx..dqdy, dzzdx, dzzdy (NY,NX).
struct DzxyArgs {
  int nx, ny, iclose;
  float dfac;
  const float* zz;
  const int *mapsta, *mapfs;
  const float *dpdx, *dpdy, *dqdx, *dqdy;
  float *dzzdx, *dzzdy;
};
void launch_wave_dzxy(const DzxyArgs& a, cudaStream_t s);

/// DISTAB: EWN1(0:n), ECG1(0:n) for n = NAR1D, each entry from WAVNU2 at depth 1.
void launch_wave_distab(int nar1d, float dsie, float ecg0, float* ewn1, float* ecg1,
                        cudaStream_t s);

/// W3CFLXY's arrays on the device: mapsf (MSEA,3); clats (0:NSEA); ecos, esin (NTH);
/// dpdx..dqdy (NY,NX); cg (0:NK+1,0:NSEA); cx, cy (0:NSEA); cflxymax (NSEA), CFLXYMAX(ISEA) at
/// cflxymax[ISEA-1].
struct CflxyArgs {
  int nsea, msea, ny, nk, nth;
  bool flcur, mgp;
  float dtg, vgx, vgy;
  const int* mapsf;
  const float *clats, *ecos, *esin, *dpdx, *dpdy, *dqdx, *dqdy, *cg, *cx, *cy;
  float* cflxymax;
};
void launch_wave_cflxy(const CflxyArgs& a, cudaStream_t s);

}  // namespace wwb
