/* oracle/dia_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * The CPU oracle of the DIA (WAVEWATCH III W3SNL1 with its INSNL1 tables), restated in plain C
 * from the reference's own C++ (ww3-gpu kokkos/src/ww_kokkos/snl1_tables.cpp:82-329 and
 * snl1_team.hpp:351-497). Only the tests, the bench's CPU-baseline leg and smoke() load it,
 * to check the CUDA library; the product library never links or calls it.
 *
 * Pinned: tests/test_oracle.py checks the float32 form against the Fortran INSNL1 tables and
 * W3SNL1 answers of the reference's frozen golden vector (tests/golden/snl1_nk25_nth24.npz)
 * and, where oracle/_ref was built from the reference's sources, against that build.
 *
 * Two forms: float32 (the reference's arithmetic, bit for bit) and float64 (the same
 * algorithm in double precision, the "FP64 DIA" that error budgets are measured against).
 * Build: oracle/Makefile, gcc -O2 -ffp-contract=off -fopenmp. */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int nk, nth;
  float xfr, dth, lam, snlc1, kdcon, kdmn, snls1, snls2, snls3, fachfe;
} oracle_snl1_config;

#define R float
#define F(name) name##f
#define S(name) name##_f32
#include "dia_body.h"
#undef R
#undef F
#undef S

#define R double
#define F(name) name
#define S(name) name##_f64
#include "dia_body.h"
#undef R
#undef F
#undef S

/* ---- exported API (ctypes) -------------------------------------------------------------- */

/* INSNL1 in float32: scal[5] = nfr, nfrhgh, nfrchg, nspecx, nspecy; wts[19] = dal1..dal3,
 * awg(8), swg(8); ipim[16 * nspecx], ic[16 * nspec], af11[nspecx] (each may be NULL, so a
 * first call with NULL tables gives the sizes). Returns 0 or -1. */
int oracle_insnl1_f32(const oracle_snl1_config *c, const float *sig, int *scal, float *wts,
                      int *ipim, int *ic, float *af11, int o0_chain) {
  tables_f32 t;
  if (insnl1_f32(c, sig, o0_chain, &t) != 0) {
    tables_free_f32(&t);
    return -1;
  }
  scal[0] = t.nfr;
  scal[1] = t.nfrhgh;
  scal[2] = t.nfrchg;
  scal[3] = t.nspecx;
  scal[4] = t.nspecy;
  wts[0] = t.dal1;
  wts[1] = t.dal2;
  wts[2] = t.dal3;
  for (int j = 0; j < 8; ++j) {
    wts[3 + j] = t.awg[j];
    wts[11 + j] = t.swg[j];
  }
  if (ipim) memcpy(ipim, t.ipim, sizeof(int) * 16 * (size_t)t.nspecx);
  if (ic) memcpy(ic, t.ic, sizeof(int) * 16 * (size_t)t.nspec);
  if (af11) memcpy(af11, t.af11, sizeof(float) * (size_t)t.nspecx);
  tables_free_f32(&t);
  return 0;
}

/* W3SNL1 on npts points, float32, OpenMP over points (nthreads <= 0: all); o0_chain as for
 * oracle_insnl1_f32. */
int oracle_w3snl1_f32(const oracle_snl1_config *c, const float *sig, int npts, const float *a,
                      const float *cg, const float *kdmean, float *s, float *d, int nthreads,
                      int o0_chain) {
  return w3snl1_batch_f32(c, sig, npts, a, cg, kdmean, s, d, nthreads, o0_chain);
}

/* The same algorithm in float64 from float64 inputs. */
int oracle_w3snl1_f64(const oracle_snl1_config *c, const double *sig, int npts, const double *a,
                      const double *cg, const double *kdmean, double *s, double *d,
                      int nthreads) {
  return w3snl1_batch_f64(c, sig, npts, a, cg, kdmean, s, d, nthreads, 0);
}
