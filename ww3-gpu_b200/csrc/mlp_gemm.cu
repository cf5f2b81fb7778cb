// ww3-gpu_b200/csrc/mlp_gemm.cu
// The surrogate MLP's GEMM on B200's fifth-generation tensor cores.
//
// One persistent CTA per SM (192 threads, about 194 KB of shared memory) walks the output tiles
// (128 x bn, bn <= 256) of C = A . B^T in a static round-robin:
//   warp 0, one lane: TMA producer. Per stage it brings a 128 x 64 tile of A and a bn x 64 tile
//     of B (bf16, 128-byte swizzle) into a 4-deep shared-memory ring, completing on the stage's
//     "full" mbarrier (cp.async.bulk.tensor, no multicast).
//   warp 1: allocates 512 TMEM columns (two fp32 accumulators of 128 lanes x 256 columns); one
//     lane issues tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulation, M=128, N=bn, K=16
//     per instruction, four per stage) and commits each stage back to the producer's "empty"
//     barrier and each finished tile to the epilogue's "tfull" barrier.
//   warps 2-5: the epilogue. Thread r of the four warps owns TMEM lane r (tile row r); it reads
//     its row 32 columns at a time (tcgen05.ld 32x32b.x32), applies the mode's bias, GELU,
//     GELU' or split-reduction add, stores, and releases the accumulator, so tile i's epilogue
//     overlaps tile i+1's MMAs in the other accumulator.
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

constexpr int kThreads = 192;
constexpr uint32_t kTileA = kBM * kBK * 2;
constexpr uint32_t kTileB = kBNMax * kBK * 2;
constexpr uint32_t kStageBytes = kTileA + kTileB;
constexpr uint32_t kTmemCols = 2 * kBNMax;
constexpr uint32_t kSpin = 1u << 24;  // polls before a wait gives up (seconds, never in a normal run)

struct Bars {
  uint64_t full[kStages];
  uint64_t empty[kStages];
  uint64_t tfull[2];
  uint64_t tempty[2];
  uint64_t drain;
  uint32_t tmem_base;
};
constexpr size_t kSmemBytes = 1024 + kStages * kStageBytes + sizeof(Bars) + 64;

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

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
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
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
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
  const float t = tanh_fast(kGeluC * (z + kGeluA * z * z * z));
  return 0.5f * z * (1.0f + t);
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

template <int MODE>
__device__ __forceinline__ void epilogue_chunk(const GemmArgs& g, int m, int n,
                                               const uint32_t (&r)[32]) {
  float v[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
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
    const float4* b4 = reinterpret_cast<const float4*>(g.bias + n);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 b = __ldg(b4 + q);
      v[4 * q + 0] += b.x;
      v[4 * q + 1] += b.y;
      v[4 * q + 2] += b.z;
      v[4 * q + 3] += b.w;
    }
    if constexpr (MODE == kEpiF32) {
      float4* o = reinterpret_cast<float4*>(g.out_f32 + row);
#pragma unroll
      for (int q = 0; q < 8; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
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
__global__ void __launch_bounds__(kThreads, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
                const GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* const smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  Bars* const bars = reinterpret_cast<Bars*>(smem + kStages * kStageBytes);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  const int m_tiles = (g.M + kBM - 1) / kBM;
  const int n_tiles = g.N / g.bn;
  const int splits = MODE == kEpiAtomic ? g.splits : 1;
  const int kb_per = g.K / kBK / splits;
  const int units = m_tiles * n_tiles * splits;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&bars->full[s], 1);
      mbar_init(&bars->empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&bars->tfull[b], 1);
      mbar_init(&bars->tempty[b], 4);  // one arrival per epilogue warp
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
          const int s = static_cast<int>(it % kStages);
          const uint32_t ph = (it / kStages) & 1u;
          if (!mbar_wait(&bars->empty[s], ph ^ 1u)) {
            ok = false;
            break;
          }
          uint8_t* const sa = smem + s * kStageBytes;
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
      for (uint32_t k = 0; k < kStages && k < issued; ++k) {
        const uint32_t last = issued - 1 - k;
        if (!mbar_wait(&bars->full[last % kStages], (last / kStages) & 1u)) atomicExch(g.err, 1);
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
          const int s = static_cast<int>(it % kStages);
          const uint32_t ph = (it / kStages) & 1u;
          if (!mbar_wait(&bars->full[s], ph)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a_addr = smem_u32(smem + s * kStageBytes);
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
    const int row = q * 32 + lane;
    uint32_t local = 0;
    bool ok = true;
    for (int u = blockIdx.x; u < units; u += gridDim.x, ++local) {
      const Unit w = decode(u, m_tiles, n_tiles);
      const uint32_t b = local & 1u, tph = (local >> 1) & 1u;
      // Warp-uniform decision: tcgen05.ld below is a warp-wide (.sync.aligned) instruction.
      if (!__all_sync(0xffffffffu, mbar_wait(&bars->tfull[b], tph))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int m = w.mt * kBM + row;
      const uint32_t tbase = tmem + (static_cast<uint32_t>(q * 32) << 16) + b * kBNMax;
      for (int c = 0; c < g.bn / 32; ++c) {
        uint32_t r[32];
        tmem_ld32(tbase + 32u * c, r);
        if (m < g.M) epilogue_chunk<MODE>(g, m, w.nt * g.bn + 32 * c, r);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars->tempty[b]);
    }
    if (!ok && lane == 0) atomicExch(g.err, 1);
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
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
  static std::once_flag once;
  std::call_once(once, [] {
    WWB_CHECK(cudaFuncSetAttribute(gemm_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kSmemBytes)));
  });
  const int m_tiles = (g.M + kBM - 1) / kBM;
  const int units = m_tiles * (g.N / g.bn) * (MODE == kEpiAtomic ? g.splits : 1);
  int sms = runtime().sm_count;
  if (sms <= 0) WWB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
  int grid = max_ctas > 0 ? max_ctas : sms;
  if (grid > units) grid = units;
  gemm_kernel<MODE><<<grid, kThreads, kSmemBytes, stream>>>(a.map, b.map, g);
  WWB_CHECK(cudaGetLastError());
}

}  // namespace

Operand make_operand(const __nv_bfloat16* base, int rows, int k, int ld, int box_rows) {
  Operand op{};
  op.rows = rows;
  op.k = k;
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
  if (g.bn != 64 && g.bn != 128 && g.bn != 192 && g.bn != 256) return no("tile width not 64/128/192/256");
  if (g.N % g.bn) return no("N not a multiple of the tile width");
  if (g.K % kBK) return no("K not a multiple of 64");
  if (a.k != g.K || b.k != g.K) return no("operand reduction length differs from K");
  if (a.rows < g.M || b.rows < g.N) return no("operand has fewer rows than the output");
  if (g.splits < 1 || (g.K / kBK) % g.splits) return no("split does not divide the K blocks");
  if (g.ldo % 8 || g.ldo < g.N) return no("output row stride not a multiple of 8 or below N");
  if (g.out_t && g.ldt < g.M) return no("transposed row stride below M");
  if (g.err == nullptr) return no("no status word");
  return true;
}

void gemm(int mode, const GemmArgs& g, const Operand& a, const Operand& b, cudaStream_t stream,
          int max_ctas) {
  switch (mode) {
    case kEpiGeluTrain: launch<kEpiGeluTrain>(g, a, b, stream, max_ctas); break;
    case kEpiGeluInfer: launch<kEpiGeluInfer>(g, a, b, stream, max_ctas); break;
    case kEpiF32: launch<kEpiF32>(g, a, b, stream, max_ctas); break;
    case kEpiDGelu: launch<kEpiDGelu>(g, a, b, stream, max_ctas); break;
    case kEpiAtomic: launch<kEpiAtomic>(g, a, b, stream, max_ctas); break;
    default: throw CudaError(cudaErrorInvalidValue, "unknown GEMM epilogue");
  }
}

}  // namespace mlp
}  // namespace wwb
