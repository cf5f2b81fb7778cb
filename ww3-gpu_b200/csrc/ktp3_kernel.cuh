// ww3-gpu_b200/csrc/ktp3_kernel.cuh
// W3KTP3 (PR3/UQ propagation in spectral space: refraction in direction and the wavenumber
// shift, with W3QCK1 and W3QCK2) on B200.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/prop_ktp3.hpp:132-353, prop_qck1.hpp, prop_qck2.hpp
// (WW3 w3pro3md.F90:1519-1961, w3uqckmd.F90 W3QCK1/W3QCK2) and the batch launcher
// kokkos/src/fortran_iface/prop3_shim.cpp:657-745.
#pragma once

#include <cuda_runtime.h>

namespace wwb {

/// W3KTP3's per-grid scalars, flags and arrays (device copies), by value into the kernel.
struct Ktp3Dev {
  int nk, nth, nspec, nk2;
  int flcth, flck, flcur;
  float dmin, ctmax, fachfa;
  const float* sig;    ///< SIG(0:NK+1)
  const float* dsip;   ///< DSIP(0:NK+1)
  const float* ecos;   ///< ECOS, ESIN, EC2, ESC, ES2 (NSPEC+NTH)
  const float* esin;
  const float* ec2;
  const float* esc;
  const float* es2;
  const int* mapwn;    ///< MAPWN(NSPEC+NTH), 1-based IK
  const int* mapth2;   ///< MAPTH2((NK+2)*NTH), 1-based VQ index
  const int* mapwn2;   ///< MAPWN2(NSPEC+NTH), 1-based VQ index
};

/// Shared memory of the kernel, bytes.
size_t ktp3_smem(const Ktp3Dev& p);

/// W3KTP3 ntimes times on npts points: va is VA(NSPEC, 0:NSEALM) (column JSEA at va +
/// JSEA*NSPEC), cg/wn are (NK+2, 0:NSEA), pscal (10, npts), jsea/isea (npts) 1-based, cflth
/// and cflk (NSEALM) written at JSEA-1. All device pointers.
void launch_ktp3(const Ktp3Dev& p, int itstep, int ntimes, float facth, float fack, int npts,
                 const int* jsea, const int* isea, const float* pscal, const float* cg,
                 const float* wn, float* va, float* cflth, float* cflk, cudaStream_t stream);

}  // namespace wwb
