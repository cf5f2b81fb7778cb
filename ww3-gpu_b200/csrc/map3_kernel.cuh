// ww3-gpu_b200/csrc/map3_kernel.cuh
// The PR3 maps on the device: W3MAP3 (MAPX2, MAPY2, MAPAXY, MAPCXY with their counters, and the
// spectral maps MAPTH2, MAPWN2) and W3MAPT (MAPTRN), so a grid change needs no host round trip.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/prop_map3.hpp:100-340 (w3map3_body, one thread in
// source order) and prop_mapt.hpp:55-79 (w3mapt_point). The maps are lists numbered by running
// counters in loop order (IX outer, IY inner, ISEA ascending); here each list is an ordered
// stream compaction: a count pass over tiles, a scan of the tile counts, and a write pass that
// ranks each tile's items in order. Every entry lands where the serial loop puts it.
#pragma once

#include <cuda_runtime.h>

namespace wwb {

/// W3MAP3's grid scalars (NX, NY, NSEA, NK, NTH, GTYPE).
struct Map3Grid {
  int nx, ny, nsea, nk, nth, gtype;
};

/// Device work of one W3MAP3 call: tile counts and offsets, the eight counters.
struct Map3Work {
  int* tiles = nullptr;   ///< 4 classes x max tiles, counts then offsets
  int* counts = nullptr;  ///< NMX0..NMX2, NMY0..NMY2, NACT, NCENT
  int* flag = nullptr;    ///< MAPTH2(1) as the call found it
  size_t tiles_n = 0;
  void release();
};

/// W3MAP3 on device arrays: mapsta (NY*NX), mapsf (NSEA,3) column-major; mapx2, mapy2, mapaxy
/// (NY*NX), mapcxy (NSEA), mapth2 ((NK+2)*NTH), mapwn2 (NSPEC+NTH). The counters go to
/// w.counts (device); the maps and counters are written only when GTYPE < 3, the spectral maps
/// only when mapth2[0] is 0, as in the reference. MAPSF must address cells of the grid.
void launch_map3(const Map3Grid& g, const int* mapsta, const int* mapsf, int* mapx2, int* mapy2,
                 int* mapaxy, int* mapcxy, int* mapth2, int* mapwn2, Map3Work& w,
                 cudaStream_t s);

/// W3MAPT on device arrays: MAPTRN(IXY) = MIN of the four transparencies of the cell < TRNMIN,
/// for the NSEA sea cells; atrnx, atrny are (NY*NX, -1:1) column-major.
void launch_mapt(int nsea, int nxy, const int* mapsf, const float* atrnx, const float* atrny,
                 int* maptrn, cudaStream_t s);

}  // namespace wwb
