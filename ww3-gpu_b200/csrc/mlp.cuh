// ww3-gpu_b200/csrc/mlp.cuh
// The learned DIA surrogate's device side: a BF16 tensor-core GEMM (tcgen05 with TMEM
// accumulators, operand tiles brought in by TMA) with the epilogues an MLP's forward and
// backward passes need, and the element-wise kernels around it (input normalisation, loss and
// output gradient, bias gradients, AdamW, the gate's per-point sums, the synthetic sea-state
// generator, the FP64 DIA that measures every surrogate result).
//
// The surrogate has no counterpart in the reference (ww3-gpu has no learned component): it is
// a faster, approximate W3SNL1 behind a per-point gate whose rejected points go back to the
// bit-exact DIA (kokkos/src/ww_kokkos/snl1_team.hpp:351-497 is the function it stands in for).
//
// Matrices are row-major with the reduction dimension contiguous ("K-major"): C[M, N] =
// A[M, K] . B[N, K]^T. A backward pass needs the transposes of activations and gradients; the
// epilogues write those copies as they store, so every GEMM reads K-major operands.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace wwb {
namespace mlp {

constexpr int kBM = 128;      ///< tile rows (one tcgen05 M=128 MMA, one TMEM lane per row)
constexpr int kBK = 64;       ///< reduction elements per pipeline stage (one 128-byte swizzle row)
constexpr int kBNMax = 256;   ///< widest tile (TMEM: two 256-column fp32 accumulators)
constexpr int kStages = 4;    ///< shared-memory pipeline depth (48 KB per stage)

/// What the epilogue does with a finished fp32 accumulator tile.
enum Epilogue : int {
  kEpiGeluTrain = 1,  ///< z = acc + bias: aux = bf16(z), out = bf16(gelu z), out_t = transpose
  kEpiGeluInfer = 2,  ///< out = bf16(gelu(acc + bias))
  kEpiF32 = 3,        ///< out_f32 = acc + bias
  kEpiDGelu = 4,      ///< g = acc * gelu'(aux): out = bf16(g), out_t = transpose
  kEpiAtomic = 5,     ///< out_f32 += acc (split reduction, red.global.add)
  kEpiSurOut = 6,     ///< the surrogate's output side: S and D of every row, gate sums (below)
  kEpiSurOutTma = 7,  ///< kEpiSurOut with tiles of 4 frequency rows (bn = 4 NTH): each 32-row
                      ///< quarter of a tile is rotated back in shared memory and stored by TMA
};

/// The original direction of canonical column j: the spectrum was rotated by the low 16 bits
/// of `packed` and, when bit 16 is set, reflected (j -> -j), so column 0 is its dominant
/// direction and columns 1..NTH/2-1 its heavier side. The DIA commutes with both (its index
/// tables are circulant in direction and symmetric under reflection).
__host__ __device__ inline int orig_col(int packed, int j, int nth) {
  const int sh = packed & 0xFFFF;
  int c = (packed >> 16) ? sh - j : sh + j;
  if (c >= nth) c -= nth;
  if (c < 0) c += nth;
  return c;
}

/// What kEpiSurOut needs besides the accumulator: per row m (a sea point) its scales ps
/// (2 NK floats: lambda, then the Hs-tendency weights) and packed direction shift; per
/// frequency row the target scale. Column i < NSPEC of row m is the normalised S of canonical
/// bin i: S(m, k NTH + orig_col(shift, j)) = (acc + bias) rowscale(k) e^lambda(k) (D, all
/// zero, is written by the caller), and the gate sums sum w v, sum w |v| (w = rowscale(k) times
/// the weight; zeroed by the caller) are added into
/// gsum[2m], gsum[2m+1]; column NSPEC is the error head, stored in head[m].
struct SurOut {
  const float* ps;
  const int* shift;
  const float* rowscale;
  float* s;
  float* d;  ///< unused by the kernel (kept for the caller's bookkeeping)
  float* head;
  float* gsum;
  int nspec, nth, nk;
};

/// One GEMM launch. Operands are described by TMA tensor maps built by make_operand().
struct GemmArgs {
  int M, N, K;          ///< C is M x N, reduction length K (multiple of kBK)
  int bn;               ///< tile columns: 64, 128, 192 or 256 (N a multiple of it)
  int splits;           ///< reduction split into this many chunks (kEpiAtomic only)
  const float* bias;    ///< N (kEpiGelu*, kEpiF32)
  __nv_bfloat16* out;   ///< M x N, row stride ldo
  __nv_bfloat16* out_t; ///< N x M, row stride ldt (may be null)
  __nv_bfloat16* aux;   ///< M x N, row stride ldo: z written (kEpiGeluTrain) or read (kEpiDGelu)
  float* out_f32;       ///< M x N, row stride ldo (kEpiF32, kEpiAtomic)
  int ldo, ldt;
  int* err;             ///< device status word: set when a bounded wait gave up
  SurOut sur;           ///< kEpiSurOut only
  int pair;             ///< 1: two CTAs of a cluster share each 256-row tile (cta_group::2); B's
                        ///< tensor map then has boxes of bn / 2 rows (gemm_b_box)
  int b_rows;           ///< kEpiSurOutTma: rows of B and entries of bias (N is padded past them;
                        ///< the padding rows of B read as zeros)
  const CUtensorMap* store;  ///< kEpiSurOutTma: host pointer to S's store map (make_store_map)
};

/// Rows of B's TMA box for this launch: bn, or bn / 2 when two CTAs share a tile.
inline int gemm_b_box(const GemmArgs& g) { return g.pair ? g.bn / 2 : g.bn; }

/// A K-major bf16 operand: `rows` rows of `k` elements, `ld` elements apart, read in boxes of
/// `box_rows` x 64 with the 128-byte swizzle the MMA's shared-memory descriptors expect.
struct Operand {
  CUtensorMap map;
  int rows, k, box;
};
Operand make_operand(const __nv_bfloat16* base, int rows, int k, int ld, int box_rows);

/// Whether the shapes suit the kernel (tile multiples, alignment); on false `why` says what.
bool gemm_shape_ok(const GemmArgs& g, const Operand& a, const Operand& b, const char** why);

/// The TMA store map of kEpiSurOutTma: S as `rows` rows of `cols` f32 (row stride `cols`),
/// written in boxes of 32 rows x `box_cols` columns.
CUtensorMap make_store_map(float* s, int rows, int cols, int box_cols);

/// Whether kEpiSurOutTma suits the surrogate's shape: bn = 4 NTH a multiple of 16 and at most
/// 256, NSPEC a multiple of bn (the error head alone in the last tile).
bool sur_tma_ok(int nk, int nth);

/// Whether a launch of epilogue `mode` with tile width `bn` fits in shared memory.
bool gemm_fits(int mode, int bn);

/// Whether g.sur is complete for a kEpiSurOut launch; on false `why` says what is missing.
bool sur_out_ok(const GemmArgs& g, const char** why);

/// C = A . B^T with epilogue `mode` on `stream` (persistent grid of at most `max_ctas` CTAs,
/// 0 = one per SM). Throws CudaError on a launch failure.
void gemm(int mode, const GemmArgs& g, const Operand& a, const Operand& b, cudaStream_t stream,
          int max_ctas = 0);

}  // namespace mlp
}  // namespace wwb
