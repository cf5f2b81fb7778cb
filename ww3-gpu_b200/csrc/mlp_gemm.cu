// ww3-gpu_b200/csrc/mlp_gemm.cu
// The surrogate MLP's GEMM on B200's fifth-generation tensor cores.
//
// One persistent CTA per SM (320 threads, up to 227 KB of shared memory) walks the output tiles
// (128 x bn, bn <= 256) of C = A . B^T in a static round-robin:
//   warp 0, one lane: TMA producer. Per stage it brings a 128 x 64 tile of A and a bn x 64 tile
//     of B (bf16, 128-byte swizzle) into a 4-deep shared-memory ring, completing on the stage's
//     "full" mbarrier (cp.async.bulk.tensor, no multicast).
//   warp 1: allocates 512 TMEM columns (two fp32 accumulators of 128 lanes x 256 columns); one
//     lane issues tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulation, M=128, N=bn, K=16
//     per instruction, four per stage) and commits each stage back to the producer's "empty"
//     barrier and each finished tile to the epilogue's "tfull" barrier.
//   warps 2-9: the epilogue, two warps per TMEM lane quarter taking alternate 32-column chunks
//     (so one warp's loads hide behind the other's work). A thread owns TMEM lane r (tile row
//     r); it reads its row 32 columns at a time (tcgen05.ld 32x32b.x32), applies the mode's
//     bias, GELU, GELU' or split-reduction add, stores (the fp32 and surrogate-output modes
//     through a shared-memory staging tile, so the stores go out row by row, coalesced), and
//     releases the accumulator, so tile i's epilogue overlaps tile i+1's MMAs in the other one.
// Every mbarrier wait is bounded: a wait that gives up sets the caller's status word, its role
// leaves its loop, and the roles it feeds give up in turn; before TMEM is freed the MMA lane
// waits for its own MMAs and the producer for its own copies, so the CTA never exits with
// tensor-core or TMA work in flight.
#include <cuda.h>

#include <cstdio>
#include <mutex>

#include "mlp.cuh"
#include "wwb_common.hpp"

namespace wwb {
namespace mlp {
namespace {

constexpr int kEpiWarps = 8;  // two per TMEM lane quarter, taking alternate 32-column chunks
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr uint32_t kTileA = kBM * kBK * 2;
constexpr uint32_t kTmemCols = 2 * kBNMax;
// The GELU-inference mode keeps the whole bias vector in shared memory, so each chunk reads its
// 32 values as 8 broadcast 16-byte loads instead of 32 shuffles (the surrogate-output mode,
// whose epilogue is shared-memory heavy already, measured slower that way and keeps shuffles).
constexpr int kBiasMax = 1536;
constexpr size_t kBiasBytes = kBiasMax * sizeof(float);
__host__ __device__ constexpr bool bias_in_smem(int mode) { return mode == 2; }
constexpr uint32_t kSpin = 1u << 24;  // polls before a wait gives up (seconds, never in a normal run)

constexpr int kStagesMax = 8;  // the paired-tile kernel's ring (its stages are half as large)

struct Bars {
  uint64_t full[kStagesMax];
  uint64_t empty[kStagesMax];
  uint64_t tfull[2];
  uint64_t tempty[2];
  uint64_t drain;
  uint32_t tmem_base;
};
static_assert(sizeof(Bars) <= 256, "barriers must fit their 256-byte slot");
// kEpiF32 and kEpiSurOut stage each epilogue warp's 32 x 32 chunk through shared memory (padded
// rows), so a thread-per-row tile is stored row by row, lane = column (coalesced); kEpiSurOut
// also keeps each row's per-frequency scale and weight for the frequency rows the tile covers.
constexpr int kStageLd = 33;
constexpr int kRowsPerTile = 8;  // frequency rows a tile of <= 256 columns covers when NTH >= 36
constexpr size_t kStageBytes32 = kEpiWarps * 32 * kStageLd * sizeof(float);
/// Epilogue warps of the single-CTA kernel per mode (a multiple of 4: one group per TMEM lane
/// quarter, the groups' warps taking every (ew / 4)-th chunk): more where the registers allow,
/// so the epilogue keeps up with the tensor cores.
__host__ __device__ constexpr int epi_warps(int mode) {
  return mode == 2 || mode == 6 || mode == 7 ? 12 : 8;
}
/// Pipeline stages of the single-CTA kernel per mode: the surrogate-output mode trades one for
/// its larger epilogue staging.
__host__ __device__ constexpr int stages_of(int mode) {
  return mode == 6 || mode == 7 ? 3 : kStages;
}
__host__ __device__ constexpr int epi_threads(int mode) { return 64 + 32 * epi_warps(mode); }
// kEpiGeluInfer stages its bf16 chunk too: 32 rows of 16 words (+1 padding word), so the warp
// stores rows of 64 contiguous bytes, eight lanes a row.
constexpr int kStageLd16 = 17;
constexpr size_t kStageBytes16 = kEpiWarps * 32 * kStageLd16 * sizeof(uint32_t);
constexpr size_t kRowConstBytes = kEpiWarps * 32 * kRowsPerTile * 2 * sizeof(float);

/// Staging bytes of `ew` epilogue warps for `mode`.
__host__ __device__ constexpr size_t stage_bytes_w(int mode, int ew) {
  return mode == 6   ? static_cast<size_t>(ew) * 32 * (kStageLd + kRowsPerTile * 2) * sizeof(float)
         : mode == 3 ? static_cast<size_t>(ew) * 32 * kStageLd * sizeof(float)
         : mode == 2 ? static_cast<size_t>(ew) * 32 * kStageLd16 * sizeof(uint32_t)
                     : 0;
}
constexpr size_t kSmemMax = 227 * 1024;

/// Bytes of one pipeline stage: the A tile and a bn-row B tile (a multiple of 1024).
__host__ __device__ constexpr uint32_t stage_bytes(int bn) {
  return kTileA + static_cast<uint32_t>(bn) * kBK * 2;
}

/// Dynamic shared memory of a launch: alignment slack, the stages, the barriers' 256-byte slot
/// and the epilogue's staging areas.
/// kEpiSurOutTma's staging: the whole 128 x bn output tile (four 32-row quarters, each the
/// dense box of one TMA store).
__host__ __device__ constexpr size_t sur_tma_stage_bytes(int bn) {
  return static_cast<size_t>(kBM) * bn * sizeof(float);
}

__host__ __device__ constexpr size_t smem_bytes(int mode, int bn) {
  return 1024 + stages_of(mode) * static_cast<size_t>(stage_bytes(bn)) + 256 +
         (mode == 7 ? sur_tma_stage_bytes(bn) : stage_bytes_w(mode, epi_warps(mode))) +
         (bias_in_smem(mode) ? kBiasBytes : 0);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

/// Wait until the phase of parity `parity` completed; false after kSpin polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < kSpin; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

/// Shared-memory matrix descriptor of a K-major tile in the 128-byte swizzle layout: rows 128 B
/// apart, 8-row groups 1024 B apart (SBO), the tile base 1024-byte aligned (base offset 0).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  return static_cast<uint64_t>((addr & 0x3FFFFu) >> 4) | (1ull << 16) |
         (static_cast<uint64_t>(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

/// Arrive on `bar` once every tcgen05.mma this thread issued so far has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// ---- kEpiSurOutTma: named barriers per TMEM lane quarter, 16-column TMEM loads, TMA stores ----
/// bar.sync on barrier `id` for `n` threads (the three epilogue warps of one lane quarter).
__device__ __forceinline__ void named_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
/// bar.red.and over barrier `id` for `n` threads: true when v is true in every one of them.
__device__ __forceinline__ bool named_and(int id, int n, bool v) {
  uint32_t out;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, %2, %3, p;\n"
      " selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(out)
      : "r"(v ? 1u : 0u), "r"(id), "r"(n)
      : "memory");
  return out != 0;
}
/// tcgen05.ld of 16 columns and its wait.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
}
/// tcgen05.ld of 16 columns without waiting (tmem_wait48 before use).
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
/// Waits for this thread's tcgen05.ld of three 16-column chunks, tied to their registers.
__device__ __forceinline__ void tmem_wait48(uint32_t (&a)[16], uint32_t (&b)[16],
                                            uint32_t (&c)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]),
                 "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]),
                 "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(b[0]), "+r"(b[1]),
                 "+r"(b[2]), "+r"(b[3]), "+r"(b[4]), "+r"(b[5]), "+r"(b[6]), "+r"(b[7]),
                 "+r"(b[8]), "+r"(b[9]), "+r"(b[10]), "+r"(b[11]), "+r"(b[12]), "+r"(b[13]),
                 "+r"(b[14]), "+r"(b[15]), "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3]),
                 "+r"(c[4]), "+r"(c[5]), "+r"(c[6]), "+r"(c[7]), "+r"(c[8]), "+r"(c[9]),
                 "+r"(c[10]), "+r"(c[11]), "+r"(c[12]), "+r"(c[13]), "+r"(c[14]), "+r"(c[15])
               :
               : "memory");
}
/// Generic-proxy writes to shared memory made visible to the TMA engine.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
/// TMA store of a box from shared memory to (x, y) of `map`; completion tracked per bulk group.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* src, int x,
                                             int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(smem_u32(src)), "r"(x), "r"(y)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
/// Until this thread's stores have read their shared memory (the staging is free again).
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
/// Until this thread's stores are complete.
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

/// tcgen05.ld of 32 columns without waiting: the registers are valid after tmem_wait32 on them.
__device__ __forceinline__ void tmem_ld32_async(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
}

/// Waits for this thread's tcgen05.ld; r (the last load's registers) is tied to the wait so no
/// use of it moves above it.
__device__ __forceinline__ void tmem_wait32(uint32_t (&r)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]),
                 "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),
                 "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]),
                 "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}

__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// GELU in its tanh form, 0.5 z (1 + tanh(c (z + 0.044715 z^3))), c = sqrt(2 / pi).
constexpr float kGeluC = 0.7978845608028654f;
constexpr float kGeluA = 0.044715f;

__device__ __forceinline__ float gelu(float z) {
  // c (z + a z^3) = z (c + c a z^2); 0.5 z (1 + t) = h + h t with h = z / 2.
  const float t = tanh_fast(z * fmaf(kGeluC * kGeluA, z * z, kGeluC));
  const float h = 0.5f * z;
  return fmaf(h, t, h);
}

__device__ __forceinline__ float dgelu(float z) {
  const float z2 = z * z;
  const float t = tanh_fast(kGeluC * (z + kGeluA * z2 * z));
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * kGeluA * z2);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

/// 32 consecutive bf16 of a row (64 bytes, 16-byte aligned).
__device__ __forceinline__ void store_row32(__nv_bfloat16* dst, const float (&v)[32]) {
  uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
  for (int q = 0; q < 4; ++q)
    d[q] = make_uint4(pack_bf16(v[8 * q + 0], v[8 * q + 1]), pack_bf16(v[8 * q + 2], v[8 * q + 3]),
                      pack_bf16(v[8 * q + 4], v[8 * q + 5]), pack_bf16(v[8 * q + 6], v[8 * q + 7]));
}

__device__ __forceinline__ void load_row32(const __nv_bfloat16* src, float (&v)[32]) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint4 u = s[q];
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const __nv_bfloat162 p = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
      const float2 f = __bfloat1622float2(p);
      v[8 * q + 2 * i] = f.x;
      v[8 * q + 2 * i + 1] = f.y;
    }
  }
}

/// Column j of the chunk into the transposed copy: 32 threads (consecutive rows m) write 64
/// contiguous bytes per column.
__device__ __forceinline__ void store_col32(__nv_bfloat16* dst_t, int ldt, int n, int m,
                                            const float (&v)[32]) {
#pragma unroll
  for (int j = 0; j < 32; ++j) dst_t[static_cast<size_t>(n + j) * ldt + m] = __float2bfloat16_rn(v[j]);
}

/// One thread's 32 columns of the other epilogues. `bl` is bias[n + lane] (the warp's lanes
/// hold the chunk's 32 bias values, read once with one coalesced load); every lane calls this,
/// rows m >= M store nothing.
template <int MODE>
__device__ __forceinline__ void epilogue_chunk(const GemmArgs& g, int m, int n,
                                               const uint32_t (&r)[32], float bl) {
  float v[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
  if constexpr (MODE == kEpiGeluTrain || MODE == kEpiGeluInfer) {
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] += __shfl_sync(0xffffffffu, bl, j);
  }
  if (m >= g.M) return;
  const size_t row = static_cast<size_t>(m) * g.ldo + n;
  if constexpr (MODE == kEpiAtomic) {
#pragma unroll
    for (int j = 0; j < 32; ++j) atomicAdd(g.out_f32 + row + j, v[j]);
    return;
  } else if constexpr (MODE == kEpiDGelu) {
    float z[32];
    load_row32(g.aux + row, z);
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = v[j] * dgelu(z[j]);
    store_row32(g.out + row, v);
    if (g.out_t) store_col32(g.out_t, g.ldt, n, m, v);
    return;
  } else {
    if constexpr (MODE == kEpiGeluTrain) store_row32(g.aux + row, v);
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = gelu(v[j]);
    store_row32(g.out + row, v);
    if constexpr (MODE == kEpiGeluTrain) {
      if (g.out_t) store_col32(g.out_t, g.ldt, n, m, v);
    }
  }
}

/// kEpiF32 through the staging tile: each thread puts its row's 32 values (plus bias) in the
/// warp's tile, then the warp stores the 32 rows one by one, 128 contiguous bytes each.
__device__ __forceinline__ void f32_chunk(const GemmArgs& g, int m_base, int n,
                                          const uint32_t (&r)[32], float bl, float* tile,
                                          int lane) {
#pragma unroll
  for (int j = 0; j < 32; ++j)
    tile[lane * kStageLd + j] = __uint_as_float(r[j]) + __shfl_sync(0xffffffffu, bl, j);
  __syncwarp();
#pragma unroll 8
  for (int rr = 0; rr < 32; ++rr) {
    const int mr = m_base + rr;
    if (mr < g.M) g.out_f32[static_cast<size_t>(mr) * g.ldo + n + lane] = tile[rr * kStageLd + lane];
  }
  __syncwarp();
}

/// kEpiGeluInfer through a bf16 staging tile: each thread packs its row's 32 GELU values into 16
/// words of the warp's tile, then eight lanes store one row's 64 contiguous bytes (four rows
/// per instruction), so every store fills whole 32-byte sectors.
__device__ __forceinline__ void gelu_infer_chunk(const GemmArgs& g, int m_base, int n,
                                                 const uint32_t (&r)[32], const float* bs,
                                                 uint32_t* tile16, int lane) {
#pragma unroll
  for (int j = 0; j < 32; j += 4) {
    const float4 b = *reinterpret_cast<const float4*>(bs + j);
    const float v0 = gelu(__uint_as_float(r[j]) + b.x);
    const float v1 = gelu(__uint_as_float(r[j + 1]) + b.y);
    const float v2 = gelu(__uint_as_float(r[j + 2]) + b.z);
    const float v3 = gelu(__uint_as_float(r[j + 3]) + b.w);
    tile16[lane * kStageLd16 + j / 2] = pack_bf16(v0, v1);
    tile16[lane * kStageLd16 + j / 2 + 1] = pack_bf16(v2, v3);
  }
  __syncwarp();
  const int sub = lane >> 3, w = 2 * (lane & 7);
#pragma unroll 4
  for (int rr = 0; rr < 32; rr += 4) {
    const int row = rr + sub;
    const int mr = m_base + row;
    const uint2 v = make_uint2(tile16[row * kStageLd16 + w], tile16[row * kStageLd16 + w + 1]);
    if (mr < g.M)
      *reinterpret_cast<uint2*>(g.out + static_cast<size_t>(mr) * g.ldo + n + 2 * w) = v;
  }
  __syncwarp();
}

/// kEpiSurOut, once per tile and thread: the scale e^lambda rowscale and the Hs-tendency weight
/// of the thread's row (sea point m) for the frequency rows k0 .. k0 + kRowsPerTile - 1, into
/// the warp's row-constant area (all loads issued before any is used).
__device__ __forceinline__ void sur_row_consts(const GemmArgs& g, int m, int k0, float* rc,
                                               int lane) {
  const SurOut& o = g.sur;
  const float* pp = o.ps + static_cast<size_t>(m < g.M ? m : 0) * 2 * o.nk;
  float lam[kRowsPerTile], wt[kRowsPerTile], rs[kRowsPerTile];
#pragma unroll
  for (int t = 0; t < kRowsPerTile; ++t) {
    const int k = k0 + t;
    const bool in = m < g.M && k < o.nk;
    lam[t] = in ? pp[k] : 0.0f;
    wt[t] = in ? pp[o.nk + k] : 0.0f;
    rs[t] = in ? __ldg(o.rowscale + k) : 0.0f;
  }
#pragma unroll
  for (int t = 0; t < kRowsPerTile; ++t) {
    rc[(lane * kRowsPerTile + t) * 2] = rs[t] * __expf(lam[t]);
    rc[(lane * kRowsPerTile + t) * 2 + 1] = rs[t] * wt[t];
  }
}

/// kEpiSurOut for one 32-column chunk of the warp's 32 rows (see SurOut in mlp.cuh). NTH >= 32,
/// so the chunk's columns lie in at most two frequency rows: columns j < jb in row k, the rest
/// in row k + 1. Each thread scales its own row's values into the warp's staging tile and adds
/// its gate sums; then the warp writes the tile out row by row, lane = column, so a sea point's
/// S stores (permuted within its frequency rows) are contiguous. (D = 0 is written by the
/// caller before the launch.)
__device__ __forceinline__ void sur_chunk(const GemmArgs& g, int m_base, int n, int k0,
                                          const uint32_t (&r)[32], float bl, int my_shift,
                                          float& racc, float& gacc, float* tile, const float* rc,
                                          int lane) {
  const SurOut& o = g.sur;
  const int k = n / o.nth;
  const int jb = (k + 1) * o.nth - n;  // first column of row k + 1 (>= 32: none)
  const float* rc0 = rc + (lane * kRowsPerTile + (k - k0)) * 2;
  const float s0 = rc0[0], w0 = rc0[1];
  const float s1 = (k - k0 + 1 < kRowsPerTile) ? rc0[2] : 0.0f;
  const float w1 = (k - k0 + 1 < kRowsPerTile) ? rc0[3] : 0.0f;
  const int valid = o.nspec - n;  // columns below NSPEC in this chunk
  if (valid >= 32) {  // the common case: every column a spectral bin
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const float v = __uint_as_float(r[j]) + __shfl_sync(0xffffffffu, bl, j);
      const bool second = j >= jb;
      const float sk = second ? s1 : s0, wk = second ? w1 : w0;
      racc += wk * v;
      gacc += wk * fabsf(v);
      tile[lane * kStageLd + j] = v * sk;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const float v = __uint_as_float(r[j]) + __shfl_sync(0xffffffffu, bl, j);
      const bool second = j >= jb;
      const float sk = second ? s1 : s0, wk = second ? w1 : w0;
      const bool in = j < valid;
      racc += in ? wk * v : 0.0f;
      gacc += in ? wk * fabsf(v) : 0.0f;
      tile[lane * kStageLd + j] = in ? v * sk : v;
    }
  }
  __syncwarp();
  // Row rr goes to S(m_base + rr, kj NTH + its own rotation of jl): lane = canonical column.
  const int i = n + lane;
  const int kj = i / o.nth, jl = i - kj * o.nth;
  const int nth = o.nth;
  float* const srow = o.s + kj * nth;
  if (valid >= 32) {
#pragma unroll 8
    for (int rr = 0; rr < 32; ++rr) {
      const int mr = m_base + rr;
      const int shr = __shfl_sync(0xffffffffu, my_shift, rr);
      const int sh = shr & 0xFFFF;
      int c = (shr >> 16) ? sh - jl : sh + jl;
      c += c < 0 ? nth : 0;
      c -= c >= nth ? nth : 0;
      if (mr < g.M) srow[static_cast<size_t>(mr) * o.nspec + c] = tile[rr * kStageLd + lane];
    }
  } else {
    const bool col_in = i < o.nspec;
    for (int rr = 0; rr < 32; ++rr) {
      const int mr = m_base + rr;
      const int shr = __shfl_sync(0xffffffffu, my_shift, rr);
      if (mr < g.M) {
        const float v = tile[rr * kStageLd + lane];
        if (col_in)
          o.s[static_cast<size_t>(mr) * o.nspec + kj * o.nth + orig_col(shr, jl, o.nth)] = v;
        else if (i == o.nspec && o.head)
          o.head[mr] = v;
      }
    }
  }
  __syncwarp();
}

/// kEpiSurOutTma's per-row inputs of one tile, loaded before the tile's accumulator is ready.
struct SurTmaRow {
  float lam[4], wt[4], rs[4], bias[3];
  int shift;
};
__device__ __forceinline__ SurTmaRow sur_tma_row(const GemmArgs& g, int m_base, int n_base, int q,
                                                 int hf, int lane) {
  const SurOut& o = g.sur;
  SurTmaRow x;
  const int m = m_base + q * 32 + lane;
  const bool in = m < g.M && n_base < o.nspec;
  const int k0 = n_base / o.nth;
  const float* pp = o.ps + static_cast<size_t>(m < g.M ? m : 0) * 2 * o.nk;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    x.lam[t] = in ? pp[k0 + t] : 0.0f;
    x.wt[t] = in ? pp[o.nk + k0 + t] : 0.0f;
    x.rs[t] = in ? __ldg(o.rowscale + k0 + t) : 0.0f;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int c0 = 16 * (hf + 3 * i);
    x.bias[i] = (lane < 16 && n_base < o.nspec && c0 < g.bn) ? __ldg(g.bias + n_base + c0 + lane)
                                                             : 0.0f;
  }
  x.shift = m < g.M ? __ldg(o.shift + m) : 0;
  return x;
}

/// One 16-column chunk of kEpiSurOutTma (tile columns c0..c0+15): bias, scale, gate sums, and
/// the rotated write into the thread's row of the staging box.
__device__ __forceinline__ void sur_tma_chunk(const uint32_t (&r)[16], int c0, int nth, float bl,
                                              const float (&sk)[4], const float (&wk)[4],
                                              int shift, float* srow, float& racc, float& gacc) {
  const int kk0 = c0 / nth;             // the chunk's first frequency row in the tile (0..3)
  const int jb = (kk0 + 1) * nth - c0;  // first column of the next frequency row
  const int jl0 = c0 - kk0 * nth;
  const float sa = kk0 == 0 ? sk[0] : kk0 == 1 ? sk[1] : kk0 == 2 ? sk[2] : sk[3];
  const float wa = kk0 == 0 ? wk[0] : kk0 == 1 ? wk[1] : kk0 == 2 ? wk[2] : wk[3];
  const float sb = kk0 == 0 ? sk[1] : kk0 == 1 ? sk[2] : kk0 == 2 ? sk[3] : 0.0f;
  const float wb = kk0 == 0 ? wk[1] : kk0 == 1 ? wk[2] : kk0 == 2 ? wk[3] : 0.0f;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float v = __uint_as_float(r[j]) + __shfl_sync(0xffffffffu, bl, j);
    const bool second = j >= jb;
    const float s = second ? sb : sa, w = second ? wb : wa;
    racc += w * v;
    gacc += w * fabsf(v);
    const int kk = second ? kk0 + 1 : kk0;
    const int jl = second ? jl0 + j - nth : jl0 + j;
    srow[kk * nth + orig_col(shift, jl, nth)] = v * s;
  }
}

/// kEpiSurOutTma for one tile (128 rows x bn = 4 NTH columns, frequency rows k0..k0+3) by the
/// three warps of TMEM lane quarter q (warp hf of them takes the 16-column chunks hf, hf+3 and
/// hf+6, loaded together): each thread (row m) adds the bias, scales its values into S's units
/// and writes them, rotated back to their directions (a permutation within each frequency row),
/// into the quarter's staging box; then one thread stores the 32 x bn box with TMA. The values
/// and the gate sums are those of kEpiSurOut (sur_chunk): the same expressions on the same
/// accumulator. The tile past NSPEC holds the error head in its first column, stored to head[m].
__device__ __forceinline__ void sur_tma_tile(const GemmArgs& g, const CUtensorMap* tc, int m_base,
                                             int n_base, uint32_t tbase, int q, int hf, int lane,
                                             float* stq, const SurTmaRow& x) {
  const SurOut& o = g.sur;
  const int nth = o.nth, bn = g.bn;
  const int m = m_base + q * 32 + lane;
  if (n_base >= o.nspec) {
    if (hf == 0) {
      uint32_t r[16];
      tmem_ld16(tbase, r);
      const float v = __uint_as_float(r[0]) + __ldg(g.bias + o.nspec);
      if (m < g.M && o.head) o.head[m] = v;
    }
    return;
  }
  float sk[4], wk[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    sk[t] = x.rs[t] * __expf(x.lam[t]);
    wk[t] = x.rs[t] * x.wt[t];
  }
  float racc = 0.0f, gacc = 0.0f;
  float* const srow = stq + lane * bn;
  const int nch = bn / 16;
  if (hf + 6 < nch) {  // three chunks (bn = 144: every warp)
    uint32_t r0[16], r1[16], r2[16];
    tmem_ld16_async(tbase + 16u * hf, r0);
    tmem_ld16_async(tbase + 16u * (hf + 3), r1);
    tmem_ld16_async(tbase + 16u * (hf + 6), r2);
    tmem_wait48(r0, r1, r2);
    sur_tma_chunk(r0, 16 * hf, nth, x.bias[0], sk, wk, x.shift, srow, racc, gacc);
    sur_tma_chunk(r1, 16 * (hf + 3), nth, x.bias[1], sk, wk, x.shift, srow, racc, gacc);
    sur_tma_chunk(r2, 16 * (hf + 6), nth, x.bias[2], sk, wk, x.shift, srow, racc, gacc);
  } else {
    for (int i = 0, c = hf; c < nch; ++i, c += 3) {
      uint32_t r[16];
      tmem_ld16(tbase + 16u * c, r);
      const float bl = i == 0 ? x.bias[0] : i == 1 ? x.bias[1] : x.bias[2];
      sur_tma_chunk(r, 16 * c, nth, bl, sk, wk, x.shift, srow, racc, gacc);
    }
  }
  fence_proxy_async_smem();
  named_sync(1 + q, 96);
  if (hf == 0 && lane == 0 && m_base + q * 32 < g.M) {
    tma_store_2d(tc, stq, n_base, m_base + q * 32);
    bulk_commit();
  }
  if (m < g.M) {
    atomicAdd(o.gsum + 2 * m, racc);
    atomicAdd(o.gsum + 2 * m + 1, gacc);
  }
}

/// The epilogue of one accumulator tile by one warp: TMEM lanes q*32.. (tile rows m_base +
/// q*32 + lane), its chunks half, half + 2, ... of the tile's bn columns from n_base.
/// Calls body(c, r) for chunks c = c0, c0 + 2, ... < nchunks with r the chunk's 32 TMEM
/// columns, the next chunk's load in flight while body runs on the current one.
template <bool DB = true, class Body>
__device__ __forceinline__ void for_chunks(uint32_t tbase, int c0, int nchunks, int step,
                                           Body&& body) {
  if constexpr (!DB) {  // one buffer: fewer registers, no load in flight during body
    for (int c = c0; c < nchunks; c += step) {
      uint32_t r[32];
      tmem_ld32_async(tbase + 32u * c, r);
      tmem_wait32(r);
      body(c, r);
    }
    return;
  }
  uint32_t ra[32], rb[32];
  int c = c0;
  if (c >= nchunks) return;
  tmem_ld32_async(tbase + 32u * c, ra);
  tmem_wait32(ra);
  for (;;) {
    if (c + step < nchunks) tmem_ld32_async(tbase + 32u * (c + step), rb);
    body(c, ra);
    c += step;
    if (c >= nchunks) break;
    tmem_wait32(rb);
    if (c + step < nchunks) tmem_ld32_async(tbase + 32u * (c + step), ra);
    body(c, rb);
    c += step;
    if (c >= nchunks) break;
    tmem_wait32(ra);
  }
}

template <int MODE>
__device__ __forceinline__ void epilogue_tile(const GemmArgs& g, int m_base, int n_base,
                                              uint32_t tbase, int q, int half, int step, int lane,
                                              float* tile, float* rowc, const float* bias_s) {
  const int row = q * 32 + lane;
  const int m = m_base + row;
  const int nchunks = g.bn / 32;
  constexpr bool kBias = MODE == kEpiGeluTrain || MODE == kEpiGeluInfer ||
                         MODE == kEpiF32 || MODE == kEpiSurOut;
  if constexpr (MODE == kEpiSurOut) {
    const int my_shift = m < g.M ? __ldg(g.sur.shift + m) : 0;
    const int k0 = n_base / g.sur.nth;
    sur_row_consts(g, m, k0, rowc, lane);
    float racc = 0.0f, gacc = 0.0f;
    for_chunks<false>(tbase, half, nchunks, step, [&](int c, const uint32_t(&r)[32]) {
      const int n = n_base + 32 * c;
      const float bl = __ldg(g.bias + n + lane);
      sur_chunk(g, m_base + q * 32, n, k0, r, bl, my_shift, racc, gacc, tile, rowc, lane);
    });
    if (m < g.M) {
      atomicAdd(g.sur.gsum + 2 * m, racc);
      atomicAdd(g.sur.gsum + 2 * m + 1, gacc);
    }
  } else if constexpr (MODE == kEpiF32) {
    for_chunks(tbase, half, nchunks, step, [&](int c, const uint32_t(&r)[32]) {
      const int n = n_base + 32 * c;
      const float bl = __ldg(g.bias + n + lane);
      f32_chunk(g, m_base + q * 32, n, r, bl, tile, lane);
    });
  } else if constexpr (MODE == kEpiGeluInfer) {
    uint32_t* const tile16 = reinterpret_cast<uint32_t*>(tile);
    for_chunks(tbase, half, nchunks, step, [&](int c, const uint32_t(&r)[32]) {
      const int n = n_base + 32 * c;
      gelu_infer_chunk(g, m_base + q * 32, n, r, bias_s + n, tile16, lane);
    });
  } else {
    for_chunks(tbase, half, nchunks, step, [&](int c, const uint32_t(&r)[32]) {
      const int n = n_base + 32 * c;
      const float bl = kBias ? __ldg(g.bias + n + lane) : 0.0f;
      epilogue_chunk<MODE>(g, m, n, r, bl);
    });
  }
}

struct Unit {
  int mt, nt, ks;
};

__device__ __forceinline__ Unit decode(int u, int m_tiles, int n_tiles) {
  Unit w;
  w.nt = u % n_tiles;
  const int rest = u / n_tiles;
  w.mt = rest % m_tiles;
  w.ks = rest / m_tiles;
  return w;
}

template <int MODE>
__global__ void __launch_bounds__(epi_threads(MODE), 1)
    gemm_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
                const __grid_constant__ CUtensorMap tc, const GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  // The 1024-byte aligned base as an offset into the shared array (not through an integer
  // cast), so the compiler keeps every derived pointer in the shared space (LDS/STS).
  uint8_t* const smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const uint32_t stage_sz = stage_bytes(g.bn);
  constexpr int ST = stages_of(MODE);
  Bars* const bars = reinterpret_cast<Bars*>(smem + ST * stage_sz);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  const int m_tiles = (g.M + kBM - 1) / kBM;
  const int n_tiles = g.N / g.bn;
  const int splits = MODE == kEpiAtomic ? g.splits : 1;
  const int kb_per = g.K / kBK / splits;
  const int units = m_tiles * n_tiles * splits;

  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&bars->full[s], 1);
      mbar_init(&bars->empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&bars->tfull[b], 1);
      mbar_init(&bars->tempty[b], epi_warps(MODE));  // one arrival per epilogue warp
    }
    mbar_init(&bars->drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&bars->tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // The bias vector after the epilogue staging (the modes that read it from shared memory).
  float* const bias_s = reinterpret_cast<float*>(
      reinterpret_cast<uint8_t*>(bars) + 256 +
      (MODE == kEpiSurOutTma ? sur_tma_stage_bytes(g.bn) : stage_bytes_w(MODE, epi_warps(MODE))));
  if constexpr (bias_in_smem(MODE))
    for (int i = threadIdx.x; i < g.N; i += blockDim.x) bias_s[i] = __ldg(g.bias + i);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = bars->tmem_base;

  if (warp == 0) {
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
      const uint32_t tx = kTileA + static_cast<uint32_t>(g.bn) * kBK * 2;
      uint32_t it = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < units && ok; u += gridDim.x) {
        const Unit w = decode(u, m_tiles, n_tiles);
        for (int kb = 0; kb < kb_per; ++kb, ++it) {
          const int s = static_cast<int>(it % ST);
          const uint32_t ph = (it / ST) & 1u;
          if (!mbar_wait(&bars->empty[s], ph ^ 1u)) {
            ok = false;
            break;
          }
          uint8_t* const sa = smem + s * stage_sz;
          mbar_expect_tx(&bars->full[s], tx);
          const int kx = (w.ks * kb_per + kb) * kBK;
          tma_load_2d(sa, &ta, &bars->full[s], kx, w.mt * kBM);
          tma_load_2d(sa + kTileA, &tb, &bars->full[s], kx, w.nt * g.bn);
        }
      }
      if (!ok) atomicExch(g.err, 1);
      // Every copy this lane started has landed before the CTA can exit (in a normal run the
      // MMA lane has already consumed them all and these waits return at once).
      const uint32_t issued = it;
      for (uint32_t k = 0; k < ST && k < issued; ++k) {
        const uint32_t last = issued - 1 - k;
        if (!mbar_wait(&bars->full[last % ST], (last / ST) & 1u)) atomicExch(g.err, 1);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // kind::f16 instruction descriptor: D f32 (bits 4-5 = 1), A and B bf16 (7-9, 10-12 = 1),
      // both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) |
                             (static_cast<uint32_t>(g.bn >> 3) << 17) |
                             (static_cast<uint32_t>(kBM >> 4) << 24);
      uint32_t it = 0, local = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < units && ok; u += gridDim.x, ++local) {
        const uint32_t b = local & 1u, tph = (local >> 1) & 1u;
        if (!mbar_wait(&bars->tempty[b], tph ^ 1u)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + b * kBNMax;
        for (int kb = 0; kb < kb_per; ++kb, ++it) {
          const int s = static_cast<int>(it % ST);
          const uint32_t ph = (it / ST) & 1u;
          if (!mbar_wait(&bars->full[s], ph)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a_addr = smem_u32(smem + s * stage_sz);
          const uint32_t b_addr = a_addr + kTileA;
#pragma unroll
          for (int j = 0; j < kBK / 16; ++j)
            umma_bf16(d, sdesc(a_addr + 32u * j), sdesc(b_addr + 32u * j), idesc,
                      (kb | j) != 0 ? 1u : 0u);
          umma_commit(&bars->empty[s]);
        }
        if (ok) umma_commit(&bars->tfull[b]);
      }
      if (!ok) atomicExch(g.err, 1);
      umma_commit(&bars->drain);
      if (!mbar_wait(&bars->drain, 0)) atomicExch(g.err, 1);
    }
  } else {
    const int q = warp & 3;  // the TMEM lane quarter this warp may read
    constexpr int EW = epi_warps(MODE);
    // Epilogue warp ew; its chunks c = ew / 4, ew / 4 + EW / 4, ...
    const int ew = warp - 2, half = ew >> 2;
    float* const tile = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(bars) + 256) +
                        static_cast<size_t>(ew) * 32 *
                            (MODE == kEpiGeluInfer ? kStageLd16 : kStageLd);
    float* const rowc = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(bars) + 256) +
                        static_cast<size_t>(EW) * 32 * kStageLd +
                        static_cast<size_t>(ew) * 32 * kRowsPerTile * 2;
    uint32_t local = 0;
    bool ok = true;
    // kEpiSurOutTma: the quarter's staging box, and its store issuer (first warp, lane 0).
    float* const stq = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(bars) + 256) +
                       static_cast<size_t>(q) * 32 * g.bn;
    const bool issuer = MODE == kEpiSurOutTma && half == 0 && lane == 0;
    for (int u = blockIdx.x; u < units; u += gridDim.x, ++local) {
      const Unit w = decode(u, m_tiles, n_tiles);
      const uint32_t b = local & 1u, tph = (local >> 1) & 1u;
      // kEpiSurOutTma: the tile's row inputs are loaded while its accumulator is computed.
      SurTmaRow xr;
      if constexpr (MODE == kEpiSurOutTma) xr = sur_tma_row(g, w.mt * kBM, w.nt * g.bn, q, half, lane);
      // Warp-uniform decision: tcgen05.ld below is a warp-wide (.sync.aligned) instruction.
      bool okw = __all_sync(0xffffffffu, mbar_wait(&bars->tfull[b], tph));
      if constexpr (MODE == kEpiSurOutTma) {
        // The quarter's three warps decide together (they share named barriers), and the
        // staging box is free once the previous tile's store has read it.
        if (issuer) bulk_wait_read();
        okw = named_and(1 + q, 96, okw);
      }
      if (!okw) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t tbase = tmem + (static_cast<uint32_t>(q * 32) << 16) + b * kBNMax;
      if constexpr (MODE == kEpiSurOutTma)
        sur_tma_tile(g, &tc, w.mt * kBM, w.nt * g.bn, tbase, q, half, lane, stq, xr);
      else
        epilogue_tile<MODE>(g, w.mt * kBM, w.nt * g.bn, tbase, q, half, EW / 4, lane, tile,
                            rowc, bias_s);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars->tempty[b]);
    }
    if (!ok && lane == 0) atomicExch(g.err, 1);
    if (issuer) bulk_wait_all();  // the tiles' stores are complete before the CTA exits
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols));
  }
}

// ------------------------------------------------------------------------------------------
// Paired tiles: two CTAs of a cluster share one 256-row output tile (cta_group::2). Each CTA
// brings its own 128 rows of A and half of the tile's bn rows of B into its shared memory, at
// the same offsets in both CTAs; the first CTA of the pair (the leader) issues one
// tcgen05.mma.cta_group::2 per K step of 16, which reads A and B from both CTAs and writes rows
// 0-127 of the accumulator into the leader's TMEM and rows 128-255 into the peer's. So each CTA
// loads 128 x 64 + bn/2 x 64 elements per stage for the same tensor-core work as a 128 x bn x 64
// stage of the single-CTA kernel: a third less shared-memory fill per flop, and stages half as
// large, so the ring is deeper. Protocol (no TMA multicast anywhere):
//   - both producers wait on their own "empty" barrier of a stage; the leader's producer posts
//     the stage's whole byte count (both CTAs' copies) on its own "full" barrier; both issue
//     their copies with .cta_group::2 so the bytes complete on the leader's "full" barrier;
//   - the leader's MMA lane waits on "full", issues, and commits with .multicast::cluster to
//     the "empty" barriers of both CTAs, and each finished tile to both CTAs' "tfull";
//   - every epilogue warp of both CTAs reads its own TMEM and arrives on the leader's "tempty"
//     (2 x 8 arrivals) through its cluster address (mapa);
//   - a cluster barrier after set-up (barriers initialised, TMEM allocated in both CTAs) and
//     before TMEM is freed, so no CTA touches a peer that has not started or has left.

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

/// The shared::cluster address of the same variable in the cluster's CTA 0.
__device__ __forceinline__ uint32_t leader_addr(const void* p) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(0));
  return r;
}

__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}

__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map,
                                                 uint32_t bar_leader, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar_leader), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void umma_bf16_pair(uint32_t d_tmem, uint64_t a, uint64_t b,
                                               uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

/// Arrive on `bar` in both CTAs of the pair once every MMA this thread issued has completed.
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
  const uint16_t mask = 0x3;
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], %1;" ::"r"(smem_u32(bar)),
      "h"(mask)
      : "memory");
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

/// Bytes of one stage of the paired kernel in each CTA: 128 rows of A and bn / 2 of B.
__host__ __device__ constexpr uint32_t pair_stage_bytes(int bn) {
  return kTileA + static_cast<uint32_t>(bn / 2) * kBK * 2;
}

__host__ __device__ constexpr size_t epi_bytes(int mode) {
  return (mode == kEpiSurOut      ? kStageBytes32 + kRowConstBytes
          : mode == kEpiF32       ? kStageBytes32
          : mode == kEpiGeluInfer ? kStageBytes16
                                  : 0) +
         (bias_in_smem(mode) ? kBiasBytes : 0);
}

/// Stages of the paired kernel's ring: as many as fit beside the epilogue's staging.
__host__ __device__ constexpr int pair_stages(int mode, int bn) {
  const size_t room = kSmemMax - 1024 - 256 - epi_bytes(mode);
  const int n = static_cast<int>(room / pair_stage_bytes(bn));
  return n > kStagesMax ? kStagesMax : n;
}

template <int MODE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    gemm_pair_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
                     const GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* const smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const uint32_t stage_sz = pair_stage_bytes(g.bn);
  const int stages = pair_stages(MODE, g.bn);
  Bars* const bars = reinterpret_cast<Bars*>(smem + stages * stage_sz);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;

  const int m_tiles = (g.M + 2 * kBM - 1) / (2 * kBM);
  const int n_tiles = g.N / g.bn;
  const int kb_per = g.K / kBK;
  const int units = m_tiles * n_tiles;
  const int cid = static_cast<int>(blockIdx.x >> 1), ncl = static_cast<int>(gridDim.x >> 1);

  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) {
      mbar_init(&bars->full[s], 1);
      mbar_init(&bars->empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&bars->tfull[b], 1);
      mbar_init(&bars->tempty[b], 2 * kEpiWarps);  // every epilogue warp of both CTAs
    }
    mbar_init(&bars->drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&bars->tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  float* const bias_s = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(bars) + 256 +
                                                 (epi_bytes(MODE) - (bias_in_smem(MODE) ? kBiasBytes : 0)));
  if constexpr (bias_in_smem(MODE))
    for (int i = threadIdx.x; i < g.N; i += blockDim.x) bias_s[i] = __ldg(g.bias + i);
  tc_fence_before();
  __syncthreads();
  cluster_sync();
  tc_fence_after();
  const uint32_t tmem = bars->tmem_base;

  if (warp == 0) {
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
      const uint32_t tx = 2 * stage_sz;  // both CTAs' copies complete on the leader's barrier
      uint32_t it = 0;
      bool ok = true;
      for (int u = cid; u < units && ok; u += ncl) {
        const Unit w = decode(u, m_tiles, n_tiles);
        for (int kb = 0; kb < kb_per; ++kb, ++it) {
          const int s = static_cast<int>(it % stages);
          const uint32_t ph = (it / stages) & 1u;
          if (!mbar_wait(&bars->empty[s], ph ^ 1u)) {
            ok = false;
            break;
          }
          uint8_t* const sa = smem + s * stage_sz;
          if (leader) mbar_expect_tx(&bars->full[s], tx);
          const uint32_t full_l = leader_addr(&bars->full[s]);
          const int kx = kb * kBK;
          tma_load_2d_pair(sa, &ta, full_l, kx, w.mt * 2 * kBM + static_cast<int>(rank) * kBM);
          tma_load_2d_pair(sa + kTileA, &tb, full_l, kx,
                           w.nt * g.bn + static_cast<int>(rank) * (g.bn / 2));
        }
      }
      if (!ok) atomicExch(g.err, 1);
      if (leader) {
        // The last stages' copies (both CTAs') have landed before the leader goes on.
        const uint32_t issued = it;
        for (uint32_t k = 0; k < static_cast<uint32_t>(stages) && k < issued; ++k) {
          const uint32_t last = issued - 1 - k;
          if (!mbar_wait(&bars->full[last % stages], (last / stages) & 1u)) atomicExch(g.err, 1);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      if (leader) {
        // kind::f16 instruction descriptor as the single-CTA kernel's, M = 256.
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) |
                               (static_cast<uint32_t>(g.bn >> 3) << 17) |
                               (static_cast<uint32_t>((2 * kBM) >> 4) << 24);
        uint32_t it = 0, local = 0;
        bool ok = true;
        for (int u = cid; u < units && ok; u += ncl, ++local) {
          const uint32_t b = local & 1u, tph = (local >> 1) & 1u;
          if (!mbar_wait(&bars->tempty[b], tph ^ 1u)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem + b * kBNMax;
          for (int kb = 0; kb < kb_per; ++kb, ++it) {
            const int s = static_cast<int>(it % stages);
            const uint32_t ph = (it / stages) & 1u;
            if (!mbar_wait(&bars->full[s], ph)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a_addr = smem_u32(smem + s * stage_sz);
            const uint32_t b_addr = a_addr + kTileA;
#pragma unroll
            for (int j = 0; j < kBK / 16; ++j)
              umma_bf16_pair(d, sdesc(a_addr + 32u * j), sdesc(b_addr + 32u * j), idesc,
                             (kb | j) != 0 ? 1u : 0u);
            umma_commit_pair(&bars->empty[s]);
          }
          if (ok) umma_commit_pair(&bars->tfull[b]);
        }
        if (!ok) atomicExch(g.err, 1);
        umma_commit_pair(&bars->drain);
      }
      // Both CTAs: every MMA (which reads this CTA's stages and writes its TMEM) has completed.
      if (!mbar_wait(&bars->drain, 0)) atomicExch(g.err, 1);
    }
  } else {
    const int q = warp & 3;
    const int ew = warp - 2, half = ew >> 2;
    float* const tile = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(bars) + 256) +
                        static_cast<size_t>(ew) * 32 *
                            (MODE == kEpiGeluInfer ? kStageLd16 : kStageLd);
    float* const rowc = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(bars) + 256 +
                                                 kStageBytes32) +
                        static_cast<size_t>(ew) * 32 * kRowsPerTile * 2;
    uint32_t local = 0;
    bool ok = true;
    for (int u = cid; u < units; u += ncl, ++local) {
      const Unit w = decode(u, m_tiles, n_tiles);
      const uint32_t b = local & 1u, tph = (local >> 1) & 1u;
      if (!__all_sync(0xffffffffu, mbar_wait(&bars->tfull[b], tph))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t tbase = tmem + (static_cast<uint32_t>(q * 32) << 16) + b * kBNMax;
      epilogue_tile<MODE>(g, w.mt * 2 * kBM + static_cast<int>(rank) * kBM, w.nt * g.bn, tbase,
                          q, half, 2, lane, tile, rowc, bias_s);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(leader_addr(&bars->tempty[b]));
    }
    if (!ok && lane == 0) atomicExch(g.err, 1);
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols));
  }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled() {
  static EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    WWB_CHECK(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000,
                                               cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || p == nullptr)
      throw CudaError(cudaErrorNotSupported, "cuTensorMapEncodeTiled entry point");
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

template <int MODE>
void launch(const GemmArgs& g, const Operand& a, const Operand& b, cudaStream_t stream,
            int max_ctas) {
  const size_t smem = smem_bytes(MODE, g.bn);
  if (smem > kSmemMax) throw CudaError(cudaErrorInvalidValue, "GEMM tile needs too much shared memory");
  static std::once_flag once;
  std::call_once(once, [] {
    WWB_CHECK(cudaFuncSetAttribute(gemm_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kSmemMax)));
  });
  const int m_tiles = (g.M + kBM - 1) / kBM;
  const int units = m_tiles * (g.N / g.bn) * (MODE == kEpiAtomic ? g.splits : 1);
  int sms = runtime().sm_count;
  if (sms <= 0) WWB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
  int grid = max_ctas > 0 ? max_ctas : sms;
  if (grid > units) grid = units;
  const CUtensorMap& tc = (MODE == kEpiSurOutTma && g.store) ? *g.store : a.map;
  gemm_kernel<MODE><<<grid, epi_threads(MODE), smem, stream>>>(a.map, b.map, tc, g);
  WWB_CHECK(cudaGetLastError());
}

template <int MODE>
void launch_pair(const GemmArgs& g, const Operand& a, const Operand& b, cudaStream_t stream) {
  const int stages = pair_stages(MODE, g.bn);
  const size_t smem = 1024 + static_cast<size_t>(stages) * pair_stage_bytes(g.bn) + 256 +
                      epi_bytes(MODE);
  if (stages < 2 || smem > kSmemMax)
    throw CudaError(cudaErrorInvalidValue, "paired GEMM tile needs too much shared memory");
  static std::once_flag once;
  std::call_once(once, [] {
    WWB_CHECK(cudaFuncSetAttribute(gemm_pair_kernel<MODE>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kSmemMax)));
  });
  const int m_tiles = (g.M + 2 * kBM - 1) / (2 * kBM);
  const int units = m_tiles * (g.N / g.bn);
  int sms = runtime().sm_count;
  if (sms <= 0) WWB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
  int clusters = sms / 2;
  if (clusters > units) clusters = units;
  if (clusters < 1) clusters = 1;
  gemm_pair_kernel<MODE><<<2 * clusters, kThreads, smem, stream>>>(a.map, b.map, g);
  WWB_CHECK(cudaGetLastError());
}

}  // namespace

Operand make_operand(const __nv_bfloat16* base, int rows, int k, int ld, int box_rows) {
  Operand op{};
  op.rows = rows;
  op.k = k;
  op.box = box_rows;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(k), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 2};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(kBK), static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_tiled()(&op.map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                                    const_cast<__nv_bfloat16*>(base), dims, strides, box, estr,
                                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError(cudaErrorInvalidValue, "cuTensorMapEncodeTiled");
  return op;
}

bool gemm_shape_ok(const GemmArgs& g, const Operand& a, const Operand& b, const char** why) {
  auto no = [&](const char* w) {
    if (why) *why = w;
    return false;
  };
  if (g.M <= 0 || g.N <= 0 || g.K <= 0) return no("empty GEMM");
  if (g.b_rows > 0) {  // kEpiSurOutTma: tiles of 4 NTH columns, B padded by the TMA unit
    if (g.bn % 16 || g.bn < 16 || g.bn > 256) return no("tile width not a multiple of 16 to 256");
    if (b.rows != g.b_rows || g.b_rows > g.N) return no("B rows differ from the declared count");
  } else {
    if (g.bn != 64 && g.bn != 128 && g.bn != 192 && g.bn != 256)
      return no("tile width not 64/128/192/256");
    if (b.rows < g.N) return no("operand has fewer rows than the output");
  }
  if (g.N % g.bn) return no("N not a multiple of the tile width");
  if (g.K % kBK) return no("K not a multiple of 64");
  if (a.k != g.K || b.k != g.K) return no("operand reduction length differs from K");
  if (a.rows < g.M) return no("operand has fewer rows than the output");
  if (g.splits < 1 || (g.K / kBK) % g.splits) return no("split does not divide the K blocks");
  if (g.ldo % 8 || g.ldo < g.N) return no("output row stride not a multiple of 8 or below N");
  if (g.out_t && g.ldt < g.M) return no("transposed row stride below M");
  if (g.err == nullptr) return no("no status word");
  if (a.box != kBM || b.box != gemm_b_box(g)) return no("operand box rows do not match the tiles");
  if (g.pair && (g.splits != 1 || g.out_t != nullptr))
    return no("paired tiles only for the inference epilogues");
  return true;
}

CUtensorMap make_store_map(float* base, int rows, int cols, int box_cols) {
  CUtensorMap map{};
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols) * 4};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(box_cols), 32u};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_tiled()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims,
                                    strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError(cudaErrorInvalidValue, "cuTensorMapEncodeTiled (S)");
  return map;
}

bool sur_tma_ok(int nk, int nth) {
  const int bn = 4 * nth;
  return nth >= 4 && bn % 16 == 0 && bn <= 256 && (nk * nth) % bn == 0 &&
         smem_bytes(kEpiSurOutTma, bn) <= kSmemMax;
}

bool gemm_fits(int mode, int bn) { return smem_bytes(mode, bn) <= kSmemMax; }

bool sur_out_ok(const GemmArgs& g, const char** why) {
  auto no = [&](const char* w) {
    if (why) *why = w;
    return false;
  };
  const SurOut& o = g.sur;
  if (!o.ps || !o.shift || !o.rowscale || !o.s || !o.gsum || !g.bias)
    return no("surrogate output: missing array");
  if (o.nth < 32 || o.nk < 1 || o.nspec != o.nk * o.nth || g.N <= o.nspec)
    return no("surrogate output: shape (NTH >= 32, an error-head column after NSPEC)");
  if ((g.bn + o.nth - 1) / o.nth + 1 > kRowsPerTile)
    return no("surrogate output: a tile covers more frequency rows than the epilogue keeps");
  return true;
}

void gemm(int mode, const GemmArgs& g, const Operand& a, const Operand& b, cudaStream_t stream,
          int max_ctas) {
  if (bias_in_smem(mode) && g.N > kBiasMax)
    throw CudaError(cudaErrorInvalidValue, "GEMM: more output columns than the bias buffer holds");
  if (g.pair) {
    switch (mode) {
      case kEpiGeluInfer: return launch_pair<kEpiGeluInfer>(g, a, b, stream);
      case kEpiF32: return launch_pair<kEpiF32>(g, a, b, stream);
      case kEpiSurOut: return launch_pair<kEpiSurOut>(g, a, b, stream);
      default: throw CudaError(cudaErrorInvalidValue, "paired tiles: inference epilogues only");
    }
  }
  switch (mode) {
    case kEpiGeluTrain: launch<kEpiGeluTrain>(g, a, b, stream, max_ctas); break;
    case kEpiGeluInfer: launch<kEpiGeluInfer>(g, a, b, stream, max_ctas); break;
    case kEpiF32: launch<kEpiF32>(g, a, b, stream, max_ctas); break;
    case kEpiDGelu: launch<kEpiDGelu>(g, a, b, stream, max_ctas); break;
    case kEpiAtomic: launch<kEpiAtomic>(g, a, b, stream, max_ctas); break;
    case kEpiSurOut: launch<kEpiSurOut>(g, a, b, stream, max_ctas); break;
    case kEpiSurOutTma:
      if (g.store == nullptr || g.pair)
        throw CudaError(cudaErrorInvalidValue, "GEMM: the TMA output epilogue needs S's store map");
      launch<kEpiSurOutTma>(g, a, b, stream, max_ctas);
      break;
    default: throw CudaError(cudaErrorInvalidValue, "unknown GEMM epilogue");
  }
}

}  // namespace mlp
}  // namespace wwb
