// ww3-gpu_b200/csrc/map3_kernel.cu
// W3MAP3 and W3MAPT on sm_100a (see map3_kernel.cuh).
//
// Each list of W3MAP3 is an ordered compaction over its loop's iteration space:
//   MAPX2, MAPAXY  (IX = 1..NX) x (IY = 2..NY-1), prop_map3.hpp:100-140, :184-204
//   MAPY2          (IX = 1..NX) x (IY = 1..NY-1), prop_map3.hpp:142-182
//   MAPCXY         ISEA = 1..NSEA,                  prop_map3.hpp:206-243
// An item belongs to one class (MAPX2's three ranges: both cells active, only the first, only
// the second; MAPCXY's central points, filled from the front, and the others, filled from the
// back) or to none. Pass 1 counts each tile's items per class, pass 2 scans the counts in tile
// order (one CTA), pass 3 ranks each tile's items in item order and writes them. An item's
// place is the number of earlier items of its class, which is the serial loop's counter.
#include "map3_kernel.cuh"

#include "wwb_common.hpp"

namespace wwb {
namespace {

constexpr int kMapBlock = 256;
constexpr int kMapItems = 8;  // consecutive items per thread
constexpr int kMapTile = kMapBlock * kMapItems;
constexpr int kScanBlock = 1024;

enum MapKind { kMapX = 0, kMapY = 1, kMapAxy = 2, kMapCxy = 3 };

struct Map3Args {
  const int* mapsta;
  const int* mapsf;
  int nx, ny, nxy, nsea;
};

template <int K>
__host__ __device__ constexpr int map_classes() {
  return K == kMapAxy ? 1 : (K == kMapCxy ? 2 : 3);
}

template <int K>
__host__ __device__ long long map_items(const Map3Args& a) {
  if (K == kMapX || K == kMapAxy) return a.ny > 2 ? static_cast<long long>(a.nx) * (a.ny - 2) : 0;
  if (K == kMapY) return a.ny > 1 ? static_cast<long long>(a.nx) * (a.ny - 1) : 0;
  return a.nsea;
}

/// MAPSTA(IY,IX) at the Fortran's column-major flat address. MAPCXY's neighbour tests can
/// address one element before or after the array (a sea point on row 1 or NY that is neither
/// a boundary nor an excluded point, which W3GRID never produces); those read 0 here.
__device__ __forceinline__ int sta(const Map3Args& a, int iy, int ix) {
  const long long i = static_cast<long long>(ix - 1) * a.ny + iy - 1;
  return (i >= 0 && i < a.nxy) ? __ldg(a.mapsta + i) : 0;
}

/// The class of item t (or -1) and the value the list stores for it.
template <int K>
__device__ __forceinline__ int map_class(const Map3Args& a, long long t, int& value) {
  if (K == kMapX || K == kMapAxy || K == kMapY) {
    const int rows = K == kMapY ? a.ny - 1 : a.ny - 2;
    const int ix = 1 + static_cast<int>(t / rows);
    const int iy = (K == kMapY ? 1 : 2) + static_cast<int>(t % rows);
    value = (ix - 1) * a.ny + iy;
    const bool c1 = sta(a, iy, ix) == 1;
    if (K == kMapAxy) return c1 ? 0 : -1;
    const bool c2 = K == kMapX ? sta(a, iy, 1 + ix % a.nx) == 1 : sta(a, iy + 1, ix) == 1;
    if (c1 && c2) return 0;
    if (c1) return 1;
    if (c2) return 2;
    return -1;
  } else {
    const int isea = static_cast<int>(t) + 1;
    value = isea;
    const int ix = __ldg(a.mapsf + (isea - 1));
    const int iy = __ldg(a.mapsf + a.nsea + (isea - 1));
    int ix0 = ix - 1, ix2 = ix + 1;
    const int iy0 = iy - 1, iy2 = iy + 1;
    if (ix == a.nx) ix2 = 1;
    if (ix == 1) ix0 = a.nx;
    const int st = sta(a, iy, ix);
    if (st == 2 || st < 0) return 1;
    const bool central = sta(a, iy0, ix0) >= 1 && sta(a, iy0, ix) >= 1 && sta(a, iy0, ix2) >= 1 &&
                         sta(a, iy, ix0) >= 1 && sta(a, iy, ix2) >= 1 && sta(a, iy2, ix0) >= 1 &&
                         sta(a, iy2, ix) >= 1 && sta(a, iy2, ix2) >= 1;
    return central ? 0 : 1;
  }
}

/// Exclusive prefix over the block of each thread's C counts; returns the block totals too.
template <int C>
__device__ __forceinline__ void block_exclusive(int (&v)[C], int (&total)[C],
                                                int (*wsum)[C]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int nw = kMapBlock / 32;
  int incl[C];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    int x = v[c];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    incl[c] = x;
    if (lane == 31) wsum[warp][c] = x;
  }
  __syncthreads();
  if (threadIdx.x < C) {
    int run = 0;
    for (int w = 0; w < nw; ++w) {
      const int x = wsum[w][threadIdx.x];
      wsum[w][threadIdx.x] = run;
      run += x;
    }
    wsum[nw][threadIdx.x] = run;
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < C; ++c) {
    total[c] = wsum[nw][c];
    v[c] = wsum[warp][c] + incl[c] - v[c];
  }
  __syncthreads();
}

template <int K>
__global__ void __launch_bounds__(kMapBlock) map_count_kernel(Map3Args a, int ntiles,
                                                              int* tiles) {
  constexpr int C = map_classes<K>();
  __shared__ int wsum[kMapBlock / 32 + 1][C];
  const long long n = map_items<K>(a);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int cnt[C];
#pragma unroll
    for (int c = 0; c < C; ++c) cnt[c] = 0;
    const long long t0 = static_cast<long long>(tile) * kMapTile + threadIdx.x * kMapItems;
#pragma unroll
    for (int k = 0; k < kMapItems; ++k) {
      const long long t = t0 + k;
      if (t < n) {
        int v;
        const int c = map_class<K>(a, t, v);
#pragma unroll
        for (int cc = 0; cc < C; ++cc) cnt[cc] += (c == cc) ? 1 : 0;
      }
    }
    int tot[C];
    block_exclusive<C>(cnt, tot, wsum);
    if (threadIdx.x < C) tiles[threadIdx.x * ntiles + tile] = tot[threadIdx.x];
  }
}

/// One CTA: the counts of each class over the tiles, in tile order, become exclusive offsets;
/// totals[c] is the class's count.
template <int C>
__global__ void __launch_bounds__(kScanBlock) map_scan_kernel(int ntiles, int* tiles,
                                                              int* totals) {
  __shared__ int wsum[kScanBlock / 32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = 0; c < C; ++c) {
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ntiles; base += kScanBlock) {
      const int i = base + threadIdx.x;
      const int v = i < ntiles ? tiles[c * ntiles + i] : 0;
      int x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wsum[warp] = x;
      __syncthreads();
      if (warp == 0) {
        int s = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, s, o);
          if (lane >= o) s += y;
        }
        wsum[lane] = s;  // inclusive over warps
      }
      __syncthreads();
      const int before = (warp > 0 ? wsum[warp - 1] : 0) + x - v;
      if (i < ntiles) tiles[c * ntiles + i] = carry + before;
      __syncthreads();
      if (threadIdx.x == 0) carry += wsum[kScanBlock / 32 - 1];
      __syncthreads();
    }
    if (threadIdx.x == 0) totals[c] = carry;
    __syncthreads();
  }
}

template <int K>
__global__ void __launch_bounds__(kMapBlock) map_write_kernel(Map3Args a, int ntiles,
                                                              const int* tiles,
                                                              const int* totals, int* out) {
  constexpr int C = map_classes<K>();
  __shared__ int wsum[kMapBlock / 32 + 1][C];
  const long long n = map_items<K>(a);
  // Where class c starts in the list: MAPX2 / MAPY2 hold their three ranges one after the
  // other; MAPCXY's second class is written from the back.
  int start[C];
  {
    int run = 0;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      start[c] = run;
      run += totals[c];
    }
  }
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int cls[kMapItems], val[kMapItems];
    int cnt[C];
#pragma unroll
    for (int c = 0; c < C; ++c) cnt[c] = 0;
    const long long t0 = static_cast<long long>(tile) * kMapTile + threadIdx.x * kMapItems;
#pragma unroll
    for (int k = 0; k < kMapItems; ++k) {
      const long long t = t0 + k;
      cls[k] = -1;
      val[k] = 0;
      if (t < n) cls[k] = map_class<K>(a, t, val[k]);
#pragma unroll
      for (int cc = 0; cc < C; ++cc) cnt[cc] += (cls[k] == cc) ? 1 : 0;
    }
    int tot[C];
    block_exclusive<C>(cnt, tot, wsum);
    int rank[C];
#pragma unroll
    for (int c = 0; c < C; ++c) rank[c] = tiles[c * ntiles + tile] + cnt[c];
#pragma unroll
    for (int k = 0; k < kMapItems; ++k) {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        if (cls[k] == c) {
          const int r = rank[c]++;
          const int pos = (K == kMapCxy && c == 1) ? a.nsea - 1 - r : start[c] + r;
          out[pos] = val[k];
        }
      }
    }
  }
}

/// The eight counters from the four lists' class totals (prop_map3.hpp:297-327).
__global__ void map3_counters_kernel(const int* tx, const int* ty, const int* ta,
                                     const int* tc, int* counts) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  counts[0] = tx[0];
  counts[1] = tx[0] + tx[1];
  counts[2] = tx[0] + tx[1] + tx[2];
  counts[3] = ty[0];
  counts[4] = ty[0] + ty[1];
  counts[5] = ty[0] + ty[1] + ty[2];
  counts[6] = ta[0];
  counts[7] = tc[0];
}

/// :434-491: MAPTH2 and MAPWN2 unless MAPTH2(1) is already set. One CTA, so the test of
/// MAPTH2(1) sees the value the call found.
__global__ void map3_spectral_kernel(int nk, int nth, int* mapth2, int* mapwn2, int* flag) {
  __shared__ int first;
  if (threadIdx.x == 0) {
    first = mapth2[0];
    *flag = first;
  }
  __syncthreads();
  if (first != 0) return;
  const int nspec = nk * nth, ld = nk + 2;
  for (int i = threadIdx.x; i < nspec; i += blockDim.x) {
    const int ik = i / nth + 1, ith = i - (ik - 1) * nth + 1;
    mapth2[i] = (ik + 1) + (ith - 1) * ld;
  }
  for (int i = threadIdx.x; i < nspec + nth; i += blockDim.x) {
    int v;
    if (i < (nk - 1) * nth) {
      const int ik = i / nth + 1, ith = i - (ik - 1) * nth + 1;
      v = (ik + 1) + (ith - 1) * ld;
    } else if (i < nspec) {
      v = nk + 1 + (i - (nk - 1) * nth) * ld;
    } else {
      v = 1 + (i - nspec) * ld;
    }
    mapwn2[i] = v;
  }
}

/// W3MAPT (prop_mapt.hpp:55-63): TRNMIN = 0.95 as its float bits; MIN as d < s ? d : s in the
/// object's operand order.
__global__ void mapt_kernel(int nsea, int nxy, const int* __restrict__ mapsf,
                            const float* __restrict__ atrnx, const float* __restrict__ atrny,
                            int* __restrict__ maptrn) {
  constexpr float kTrnMin = 0x1.e66666p-1f;
  auto mn = [](float d, float s) { return d < s ? d : s; };
  for (int isea = 1 + blockIdx.x * blockDim.x + threadIdx.x; isea <= nsea;
       isea += gridDim.x * blockDim.x) {
    const int ixy = mapsf[2 * nsea + isea - 1];
    const float my = mn(atrny[(ixy - 1) + 2 * nxy], atrny[ixy - 1]);
    const float mx = mn(atrnx[(ixy - 1) + 2 * nxy], atrnx[ixy - 1]);
    const float m = mn(my, mx);
    maptrn[ixy - 1] = (m < kTrnMin) ? 1 : 0;
  }
}

int tiles_of(long long n) { return static_cast<int>((n + kMapTile - 1) / kMapTile); }

template <int K>
void run_list(const Map3Args& a, int* tiles, int* totals, int* out, cudaStream_t s) {
  const int nt = tiles_of(map_items<K>(a));
  if (nt == 0) {
    WWB_CHECK(cudaMemsetAsync(totals, 0, sizeof(int) * map_classes<K>(), s));
    return;
  }
  map_count_kernel<K><<<nt, kMapBlock, 0, s>>>(a, nt, tiles);
  map_scan_kernel<map_classes<K>()><<<1, kScanBlock, 0, s>>>(nt, tiles, totals);
  map_write_kernel<K><<<nt, kMapBlock, 0, s>>>(a, nt, tiles, totals, out);
  WWB_CHECK(cudaGetLastError());
}

}  // namespace

void Map3Work::release() {
  if (tiles) cudaFree(tiles);
  if (counts) cudaFree(counts);
  tiles = nullptr;
  counts = nullptr;
  flag = nullptr;
  tiles_n = 0;
}

void launch_map3(const Map3Grid& g, const int* mapsta, const int* mapsf, int* mapx2, int* mapy2,
                 int* mapaxy, int* mapcxy, int* mapth2, int* mapwn2, Map3Work& w,
                 cudaStream_t s) {
  const Map3Args a{mapsta, mapsf, g.nx, g.ny, g.nx * g.ny, g.nsea};
  // Tile counts of the four lists side by side (3 + 3 + 1 + 2 classes), then 4 x 3 totals.
  const int tx = tiles_of(map_items<kMapX>(a)), ty = tiles_of(map_items<kMapY>(a));
  const int tc = tiles_of(map_items<kMapCxy>(a));
  const size_t need = static_cast<size_t>(3 * tx + 3 * ty + tx + 2 * tc) + 16;
  if (w.counts == nullptr) {
    WWB_CHECK(cudaMalloc(&w.counts, sizeof(int) * 16));
    w.flag = w.counts + 8;
  }
  if (need > w.tiles_n) {
    WWB_CHECK(cudaStreamSynchronize(s));
    if (w.tiles) WWB_CHECK(cudaFree(w.tiles));
    w.tiles = nullptr;
    w.tiles_n = 0;
    WWB_CHECK(cudaMalloc(&w.tiles, sizeof(int) * need));
    w.tiles_n = need;
  }
  if (g.gtype < 3) {
    int* const t_x = w.tiles;
    int* const t_y = t_x + 3 * tx;
    int* const t_a = t_y + 3 * ty;
    int* const t_c = t_a + tx;
    int* const tot = t_c + 2 * tc;  // 12 ints: X, Y, AXY, CXY
    run_list<kMapX>(a, t_x, tot, mapx2, s);
    run_list<kMapY>(a, t_y, tot + 3, mapy2, s);
    run_list<kMapAxy>(a, t_a, tot + 6, mapaxy, s);
    run_list<kMapCxy>(a, t_c, tot + 9, mapcxy, s);
    map3_counters_kernel<<<1, 32, 0, s>>>(tot, tot + 3, tot + 6, tot + 9, w.counts);
    WWB_CHECK(cudaGetLastError());
  }
  map3_spectral_kernel<<<1, 256, 0, s>>>(g.nk, g.nth, mapth2, mapwn2, w.flag);
  WWB_CHECK(cudaGetLastError());
}

void launch_mapt(int nsea, int nxy, const int* mapsf, const float* atrnx, const float* atrny,
                 int* maptrn, cudaStream_t s) {
  if (nsea <= 0) return;
  const int blocks = (nsea + 255) / 256;
  mapt_kernel<<<blocks < 4096 ? blocks : 4096, 256, 0, s>>>(nsea, nxy, mapsf, atrnx, atrny,
                                                              maptrn);
  WWB_CHECK(cudaGetLastError());
}

}  // namespace wwb
