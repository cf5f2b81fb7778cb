// ww3-gpu_b200/csrc/mlp_ops.cuh
// The surrogate's element-wise device work around the tensor-core GEMM: synthetic sea states,
// the spectrum normalisation (input side) and its inverse (output side, with the gate), the
// training loss and output gradient, bias gradients, transposes, AdamW, and the FP64 DIA that
// every surrogate result is measured against.
//
// Normalisation. W3SNL1 (kokkos/src/ww_kokkos/snl1_team.hpp:383-496) computes, per point,
//   S(k, th) = CONS(kdmean) * CONX(k) * G(UE)(k, th),  UE = A / CONX,  CONX = CG / (2 pi sigma),
// with G a cubic form of UE whose terms at row k carry AF11 = f^11 of rows near k (sections
// 3-4). So S(k, .) scales, point by point and row by row, as
//   e^lambda(k) = CONS * CONX(k) * AF11(k) * u(k)^3,  u(k) = the largest UE within 3 rows of k,
// and T = S / (e^lambda(k) rowscale(k)) is of order one in every row of every spectrum (rowscale
// the per-row RMS of S e^-lambda over the first chunk of the training set). The network maps
// the spectrum's shape to T; depth (CONX, CONS), amplitude and the steep frequency dependence
// are applied exactly outside it. Directions are rotated so the spectrum's dominant direction
// comes first (the DIA commutes with a cyclic shift of directions, its index tables being
// circulant in direction), and the rotation is undone on the output. Network input:
// ln(UE / max UE + 1e-6) / 7 + 1 per bin, then ln(kdmean) / 5 and CONS / SNLC1 - 1.
//
// Per point the normalisation keeps 2 NK floats ("ps"): lambda(k), then the weight of row k in
// the Hs tendency, e^lambda(k) DDEN(k) / CG(k) divided by its largest value (DDEN = DTH DSII SIG,
// DSII = SIG (XFR - 1/XFR) / 2).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace wwb {
namespace mlp {

/// Per-grid constants of the surrogate's pre- and post-processing.
struct SurGrid {
  int nk, nth, nspec;
  int din, dout;          ///< padded network widths (multiples of 64)
  const float* sig;       ///< device, NK
  const float* rowscale;  ///< device, NK: RMS of the scaled targets per frequency row
  float snlc1, kdcon, kdmn, snls1, snls2, snls3;
  float dth, xfr;
};

/// Sea-state draw of the synthetic training and test sets (JONSWAP wind sea with cos^2s
/// spreading, optionally a swell system), seeded per point.
struct SynthDraw {
  uint64_t seed;
  double bimodal;    ///< fraction of points with an added swell system
  double dmin, dmax; ///< depth drawn log-uniformly in [dmin, dmax] (dmin == dmax: fixed)
};

/// Gate thresholds: a point keeps the surrogate's S when the energy residual of its output
/// |sum w S| / sum w |S| (w = DDEN / CG, the Hs-tendency weight) is at most `energy` and the
/// network's own predicted error (the log of its Hs-tendency error, output column NSPEC) is at
/// most `log_err`.
struct GateParams {
  float energy;
  float log_err;
};

void synth(const SurGrid& g, const SynthDraw& d, long long p0, int npts, float* a, float* cg,
           float* kdmean, cudaStream_t st);

/// Network input rows x (npts x ldx bf16), the per-point scales ps (npts x 2 NK) and the
/// direction shift; with dzero (npts x NSPEC) and gzero (npts x 2) non-null, also zeros there
/// (the gated path's D and gate sums).
void prep(const SurGrid& g, int npts, const float* a, const float* cg, const float* kdmean,
          __nv_bfloat16* x, int ldx, float* ps, int* shift, cudaStream_t st,
          float* dzero = nullptr, float* gzero = nullptr);

/// Accumulate sum over points and directions of (S e^-lambda)^2 per row into acc (double, NK,
/// zeroed by the caller), and count the points with a nonempty spectrum into cnt.
void rowscale_acc(const SurGrid& g, int npts, const float* s, const float* ps, double* acc,
                  unsigned long long* cnt, cudaStream_t st);

/// Normalised targets t (npts x ldt fp32) from the DIA's S.
void targets(const SurGrid& g, int npts, const float* s, const float* ps, const int* shift,
             float* t, int ldt, cudaStream_t st);

/// The gate of every point after the fused output epilogue (kEpiSurOut): from its gate sums
/// (gsum, 2 per point) and head output, accept or add it to the compacted rejected list
/// (count at *nrej, zeroed by the caller; also added to *nrej_total when given; a point's entry
/// is base + its index, so several chunks can fill one list); per-point flag and (gv, may be
/// null) head and energy residual.
void gate_points(const GateParams& gate, int npts, const float* gsum, const float* head,
                 int* accepted, float* gv, int* rej_list, int* nrej, int* nrej_total,
                 cudaStream_t st, int base = 0);

/// The rows of `rows` (a list of *count entries) of src (rows of `width` floats) packed into
/// dst, at most `cap` of them, with the list's entries into list_dst and *count into count_dst:
/// the rejected points' D of one chunk, for a copy to the host of those rows alone.
void gather_listed_rows(const int* count, const int* rows, int cap, int width, const float* src,
                        float* dst, int* list_dst, int* count_dst, cudaStream_t st);

/// Training loss and the output gradient. out (m x ldo fp32), t (m x ldt): grad (m x dout bf16)
/// = dL/dout; loss (3 floats: MSE, energy-budget, error-head terms) accumulated.
struct LossWeights {
  float mu;      ///< weight of the squared relative Hs-tendency error
  float lambda;  ///< weight of the error head
  int head;      ///< 1: column NSPEC is trained as the error head
};
/// ps (m x 2 NK, may be null: no energy term) gives each row's Hs-tendency weights.
void loss_grad(const SurGrid& g, const LossWeights& w, int m, int nvalid, const float* out,
               int ldo, const float* t, int ldt, const float* ps, __nv_bfloat16* grad, int ldg,
               float* loss, cudaStream_t st);

/// Batch rows r < m of the training set: x, t and ps rows idx(r), idx(r) a seeded draw in
/// [0, n) (or r + offset when seed == 0).
void gather_batch(int m, long long n, uint64_t seed, long long offset, const __nv_bfloat16* xs,
                  int ldx, const float* ts, int ldt, const float* pss, int ldp,
                  __nv_bfloat16* xb, float* tb, float* psb, cudaStream_t st);

/// dst (cols x rows) = src (rows x cols)^T, bf16; ld's in elements.
void transpose(const __nv_bfloat16* src, int rows, int cols, int lds, __nv_bfloat16* dst, int ldd,
               cudaStream_t st);

/// db[n] = sum over m of gt[n][m] (gt is the transposed gradient, n rows of m).
void colsum(const __nv_bfloat16* gt, int n, int m, int ldt, float* db, cudaStream_t st);

/// AdamW on one weight matrix (n x k) and its bias: fp32 master w, moments m, v, gradient g
/// (zeroed after use), the bf16 copy wb (n x k) and its transpose wt (k x n).
struct Adam {
  float lr, beta1, beta2, eps, wd;
  float c1, c2;  ///< bias corrections 1 - beta^t
};
void adamw(const Adam& h, int n, int k, float* w, float* m, float* v, float* g,
           __nv_bfloat16* wb, __nv_bfloat16* wt, cudaStream_t st);
void adamw_vec(const Adam& h, int n, float* w, float* m, float* v, const float* g,
               cudaStream_t st);

/// Weights U(-a, a), a = gain * sqrt(3 / fan_in), rows >= nrows_valid zero; fp32 and bf16 copies.
void init_weights(uint64_t seed, int n, int k, int nrows_valid, float gain, float* w,
                  __nv_bfloat16* wb, __nv_bfloat16* wt, cudaStream_t st);
void to_bf16(const float* w, int n, int k, __nv_bfloat16* wb, __nv_bfloat16* wt, cudaStream_t st);

/// The FP64 DIA (the same four sections as W3SNL1 in double precision, tables in double) and
/// the error of a candidate S against it, per point, as 10 doubles:
///   0 Hs, 1 Hs tendency of the FP64 S, 2 Hs tendency of the candidate, 3 gross Hs tendency
///   (sum of |S| terms), 4 sum |band tendency error|, 5 sum |band tendency|, 6 sum (S - S64)^2,
///   7 sum S64^2, 8 mean-frequency tendency of the FP64 S, 9 of the candidate.
struct DiaF64 {
  int nk, nth, nfr, nfrhgh, nfrchg, nspec, nspecx;
  double dal1, dal2, dal3, awg[8], swg[8];
  double snlc1, kdcon, kdmn, snls1, snls2, snls3, fachfe, dth, xfr;
  const int* ipim;       ///< device, 16 x NSPECX
  const int* ic;         ///< device, 16 x NSPEC
  const double* af11;    ///< device, NFRCHG (per row)
  const double* sig;     ///< device, NK
};
size_t dia_f64_smem(const DiaF64& t);
void dia_f64_judge(const DiaF64& t, int npts, const float* a, const float* cg,
                   const float* kdmean, const float* s_cand, double* stats, double* s64,
                   double* d64, cudaStream_t st);

}  // namespace mlp
}  // namespace wwb
