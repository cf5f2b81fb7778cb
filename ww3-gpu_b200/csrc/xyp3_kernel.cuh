// ww3-gpu_b200/csrc/xyp3_kernel.cuh
// W3XYP3 with W3QCK3 (PR3/UQ spatial propagation) and W3GATH/W3SCAT on B200, for a chunk of
// spectral components at once.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/prop_xyp3.hpp:155-584, prop_qck3.hpp:60-224,
// prop_params.hpp:47-171 (WW3 w3pro3md.F90:641-1477, w3uqckmd.F90 W3QCK3) and the batch
// launcher kokkos/src/fortran_iface/prop3_shim.cpp:477-660.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace wwb {

/// Per-call grid data on the device (all arrays as W3XYP3 reads them, 0-based pointers).
struct Xyp3Grid {
  int nx, ny, nsea, nk, nth, nspec, iclose, flcx, flcy, flagll, flcur;
  float dtcfl, dth, xfr, wdcg, wdth;
  int nmx0, nmx1, nmx2, nmy0, nmy1, nmy2, nact, ncent;
  int global;                       ///< ICLOSE /= ICLOSE_NONE
  const int* mapsf;                 ///< (NSEA, 3)
  const float* clats;               ///< (0:NSEA)
  const float* sig;                 ///< (0:NK+1)
  const float* ecos;                ///< (NSPEC+NTH)
  const float* esin;
  const float *dpdx, *dpdy, *dqdx, *dqdy, *gsqrt;  ///< (NY, NX)
  const float* atrnx;               ///< (NY*NX, -1:1)
  const float* atrny;
  const int *mapx2, *mapy2, *mapaxy;  ///< (NY*NX)
  const int* mapsta;                ///< (NY*NX), the dummy W3XYP3 and W3SCAT get
  const int* maptrn;                ///< (NY*NX), 0/1
  const int* mapstx;                ///< MAPSTX(1-2*NY : NY*(NX+2)), built per call
  const int* cell_sea;              ///< ISEA of cell IXY (0 for land), NY*NX
  const int* sea_pos;               ///< position (1-based) of ISEA in MAPCXY, NSEA
  const int* bnd_last;              ///< IBI of the last ISBPI entry naming ISEA, or 0; NSEA
  /// Per cell IXY (NY*NX), or null: bits 0-1 the kind of the x face at IXY in MAPX2 (0 none,
  /// 1 interior, 2 boundary with the CFL at IXY, 3 boundary with the CFL at IXY+INC), bits 2-3
  /// the same for MAPY2, bit 4 set when IXY is in MAPAXY. Null when a list names a cell twice:
  /// the sweeps then run as list kernels.
  const unsigned char* cell_kind;
  /// Per cell T of FIELD (NY*(NX+3), T = 1-NY .. NY*(NX+2) at T+NY-1), or null: the sea points
  /// whose averaging statements can reach T (T - D(j), D = 0, 1, -1, NY, -NY, NY+1, NY-1,
  /// -NY+1, -NY-1), as 4-bit j in the averaging loop's order (their MAPCXY positions), 0xF
  /// after the last; built once per call (launch_xyp3_gather_order). With it the averaging
  /// runs tiled (average_tile_kernel); it needs cell_kind and NY >= 3.
  unsigned long long* gather_order;
  const float* cg;                  ///< (0:NK+1, 0:NSEA)
  const float* cx;                  ///< (0:NSEA)
  const float* cy;
  const float* bbpi0;               ///< (NSPEC, 0:NBI)
  const float* bbpin;
  int flbpi, nbi;
  float dsec_day, dsec_bpi0, dsec_bpin, dtg;
  float cxmin, cxmax, cymin, cymax;  ///< MINVAL/MAXVAL of CX, CY over the sea (FLCUR)
  // W3_MPI (naproc > 0): sea point ISEA is column K = (ISEA-1)/NAPROC + 1 of rank
  // IP = MOD(ISEA-1,NAPROC) + 1. This rank's points are VA columns; another rank's value of the
  // L-th listed component is rbuf[poff[IP-1] + L*NSEALM + K-1] (W3GATH's GSTORE) and W3SCAT's
  // SSTORE goes to the same place of sbuf. naproc == 0: W3_SHRD, column ISEA of VA.
  int naproc, iaproc, nsealm;
  const int* poff;
  const float* rbuf;
  float* sbuf;
};

/// One chunk of components: their indices and the device work arrays (component-major).
struct Xyp3Chunk {
  int ncomp;
  int l0;             ///< place of the chunk's first component in the list of all components
  const int* isp;     ///< 1-based ISP of each component
  float* vq;          ///< ncomp x NQ, NQ = NY*(NX+3): FIELD(1-NY : NY*(NX+2))
  float* aq;          ///< ncomp x NQ
  float* vlcflx;      ///< ncomp x NY*(NX+1)
  float* vlcfly;      ///< ncomp x NY*(NX+1)
  float* fla;         ///< ncomp x NY*(NX+1): FLA(1-NY : NY*NX)
  float* rdi;         ///< ncomp x 4 x NSEA
  int* iixy;          ///< ncomp x 4 x NSEA
  unsigned* tcode;    ///< ncomp x NSEA: the cells of each point's 8 averaging statements
  struct Comp* comp;  ///< ncomp per-component constants (device)
};

/// Bytes of work storage per component.
size_t xyp3_bytes_per_component(const Xyp3Grid& g);

/// Bytes of one component's constants (the chunk's comp array holds one per component).
size_t xyp3_comp_bytes();

/// W3GATH, W3XYP3 and W3SCAT for every component of the chunk, on the resident VA
/// (NSPEC, 0:NSEALM) va. The chunk's arrays must be allocated (xyp3_bytes_per_component).
void run_xyp3_chunk(const Xyp3Grid& g, Xyp3Chunk& c, float* va, cudaStream_t s);

/// The first half of run_xyp3_chunk: the components' constants (sub-step counts, rotated
/// speeds) into the chunk's device array; returns the largest sub-step count (synchronises).
int setup_xyp3_chunk(const Xyp3Grid& g, Xyp3Chunk& c, cudaStream_t s);

/// The second half: one propagation of the chunk's components on va with ntmax sub-steps,
/// launches only (no host synchronisation, no host memory), so a stream capture can record it.
void launch_xyp3_chunk(const Xyp3Grid& g, const Xyp3Chunk& c, float* va, int ntmax,
                       cudaStream_t s);

/// ww_xyp3_mpi_pack (unpack false): buf[J*NSEALM + K-1] = VA(ISPS(J+1), K), K = 1 .. NSEALM;
/// ww_xyp3_mpi_unpack (unpack true) the other way. d_isps holds nisp 1-based components.
void launch_va_components(bool unpack, float* va, int nspec, int nsealm, const int* isps,
                          int nisp, float* buf, cudaStream_t s);

/// MINVAL/MAXVAL of CX(1:NSEA), CY(1:NSEA) as gfortran evaluates them (NaN entries skipped,
/// NaN when all are NaN, +-HUGE when empty), into g.cxmin .. g.cymax.
void xyp3_current_range(Xyp3Grid& g, cudaStream_t s);

/// Fills g.gather_order (allocated, NY*(NX+3) words) on stream s.
void launch_xyp3_gather_order(const Xyp3Grid& g, cudaStream_t s);

}  // namespace wwb
