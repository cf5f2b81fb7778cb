/* include/ww_b200.h -- the C ABI of libww_b200.so.
 *
 * libww_b200.so is a drop-in for the C ABI that the WAVEWATCH III fork's run-time switch binds
 * (ww3-gpu's kokkos/src/fortran_iface/ww_kokkos_c.hpp, resident_c.hpp and prop3_c.hpp): the
 * same symbol names, argument order, Fortran column-major layouts and status codes, backed by
 * hand-written CUDA kernels for B200 (sm_100a). Each declaration cites the reference entry it
 * replaces. Entries marked "B200 extension" have no counterpart in the reference.
 *
 * Rules carried over from the reference ABI (ww_kokkos_c.hpp:6-33):
 *  1. Arrays are Fortran-ordered (column-major), caller-owned and borrowed for the call.
 *  2. float is WW3's default REAL; LOGICAL crosses as int 0/1.
 *  3. Nothing throws across the boundary. Entries return or record a WwKokkosStatus, read back
 *     with the part's *_last_error(); each failure prints one line to stderr. On a validation
 *     failure nothing is written through output pointers. npts == 0 is a no-op.
 *  4. Not thread-safe: one caller at a time. Contexts are kept per grid index `igrid`.
 * The device is chosen by WW_KOKKOS_DEVICE_ID (default 0); the communicator is ignored.
 */
#ifndef WW_B200_H
#define WW_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: ww_kokkos_c.hpp:42-50 (same values). */
enum WwKokkosStatus {
  WW_KOKKOS_OK = 0,
  WW_KOKKOS_ERR_NOT_INITIALISED = 1,
  WW_KOKKOS_ERR_BAD_SHAPE = 2,
  WW_KOKKOS_ERR_KERNEL = 3,
  WW_KOKKOS_ERR_RUNTIME = 4,
  WW_KOKKOS_ERR_UNSUPPORTED = 5,
  WW_KOKKOS_ERR_TABLE = 6
};

/* ---------------------------------------------------------------- runtime */

/* Replaces ww_kokkos_init (ww_kokkos_c.hpp:73): selects the CUDA device from
 * WW_KOKKOS_DEVICE_ID, creates the library's streams, reads the run-time flags. Idempotent.
 * Returns WW_KOKKOS_OK or WW_KOKKOS_ERR_RUNTIME (no usable CUDA device). */
int ww_kokkos_init(int comm_f);

/* Replaces ww_kokkos_finalize (ww_kokkos_c.hpp:79): frees every grid context and stream. Safe
 * to call twice or before init. */
void ww_kokkos_finalize(void);

/* ---------------------------------------------------------------- W3SNL1 (the DIA) */

/* Replaces ww_snl1_init (ww_kokkos_c.hpp:98-100): builds the INSNL1 tables of grid `igrid` on
 * the host (the reference's snl1_tables.cpp:82-329 arithmetic) and uploads them. `sig` is
 * SIG(1:nk), copied. Returns OK, NOT_INITIALISED, BAD_SHAPE or RUNTIME; on failure the grid is
 * left unconfigured. */
int ww_snl1_init(int igrid, int nk, int nth, float xfr, float dth, float lam, float snlc1,
                 float kdcon, float kdmn, float snls1, float snls2, float snls3, float fachfe,
                 const float* sig);

/* B200 extension. Configures grid `igrid` from INSNL1 tables the caller already holds (WW3's
 * own W3ADATMD arrays, so the device uses the Fortran build's exact AF11 bits), instead of
 * rebuilding them. Same scalars as ww_snl1_init, then: scal[5] = NFR, NFRHGH, NFRCHG, NSPECX,
 * NSPECY; wts[19] = DAL1..DAL3, AWG1..AWG8, SWG1..SWG8; ipim[16*NSPECX] = IP11..IP14,
 * IM11..IM14, IP21..IP24, IM21..IM24; ic[16*NSPEC] = IC11, IC21 .. IC81, IC12 .. IC82;
 * af11[NSPECX]. Index entries are 0-based (Fortran value minus one). Returns OK,
 * NOT_INITIALISED, BAD_SHAPE (inconsistent sizes or an entry out of range) or RUNTIME. */
int ww_snl1_init_tables(int igrid, int nk, int nth, float xfr, float dth, float lam,
                        float snlc1, float kdcon, float kdmn, float snls1, float snls2,
                        float snls3, float fachfe, const float* sig, const int* scal,
                        const float* wts, const int* ipim, const int* ic, const float* af11);

/* Replaces ww_snl1 (ww_kokkos_c.hpp:115-116): W3SNL1 for npts sea points from host memory.
 * a, s, d are (nspec, npts), cg (nk, npts), kdmean (npts). s and d are overwritten. The copies
 * in and out are pipelined with the kernel in chunks; page-locked caller memory copies fastest.
 * Status in ww_snl1_last_error(). */
void ww_snl1(int igrid, int npts, const float* a, const float* cg, const float* kdmean,
             float* s, float* d);

/* B200 extension. W3SNL1 on device-resident arrays (same shapes as ww_snl1), launched on the
 * CUDA stream `stream` (a cudaStream_t; NULL is the legacy default stream) without any copy or
 * synchronisation. Status in ww_snl1_last_error(); launch errors are reported, execution errors
 * surface at the caller's next synchronisation. */
void ww_snl1_device(int igrid, int npts, const float* a, const float* cg, const float* kdmean,
                    float* s, float* d, void* stream);

/* B200 extension; no counterpart in the reference. ww_snl1 (same arguments, results and status
 * in ww_snl1_last_error) for a caller that must not allocate device memory once its set-up is
 * over: a coupled run whose partner component has already reserved the rest of HBM through its
 * own pool, so a late cudaMalloc would fail mid-run, or an operational forecast whose device
 * footprint is fixed at start-up so that an out-of-memory cannot end it hours later, and where
 * a cudaFree would stall the other components' work on the device. The copies go through one
 * 32 MiB static device array instead of per-grid buffers: npts is limited by
 * 3*c(npts*NSPEC) + c(npts*NK) + c(npts) <= 8388608 floats, c() rounding up to a multiple of
 * 64 (2137 points of a 36x36 grid); a larger npts is ERR_BAD_SHAPE with nothing written. The
 * first call on a device does the set-up (resolves the array's address); make it before any
 * stream capture. The device current at the call must be the one of the grid's ww_snl1_init
 * (else ERR_BAD_SHAPE, nothing written). The array is one per device for the whole process:
 * calls that overlap in time (several host threads) race on it. No cudaMalloc, cudaFree or
 * allocating library call. */
void ww_snl1_noalloc(int igrid, int npts, const float* a, const float* cg, const float* kdmean,
                     float* s, float* d);

/* Replaces ww_snl1_enabled (ww_kokkos_c.hpp:120): 1 if WW_KOKKOS_SNL1 resolves to on (see
 * ww_kokkos_flag) at ww_kokkos_init, else 0. */
int ww_snl1_enabled(void);

/* Replaces ww_snl1_last_error (ww_kokkos_c.hpp:133). */
int ww_snl1_last_error(void);

/* B200 extension: the table builders of the GQM form of NL1 (INSNLGQM's helpers, w3snl1md.F90
 * :1185-1500; the reference's host C++ snl1_couple.hpp, snl1_gauleg.hpp, snl1_f1f1f1.hpp, which
 * it exports through no C entry), bit for bit as the reference computes them.
 * ww_snl1_gqm_couple: COUPLE, the Webb four-wave coupling coefficient, in FP64 on the device for
 * n quadruplets; k is (8, n) column-major (XK1, YK1, XK2, YK2, XK3, YK3, XK4, YK4 per column),
 * coef (n) out, diag (n) out or NULL: bits 1/2 (term 1-3 is 0/0 / infinite) and 4/8 (term
 * 1-4), the Fortran's warnings, the term left out. OK, NOT_INITIALISED, BAD_SHAPE, KERNEL.
 * ww_snl1_gqm_gauleg: GAULEG on the host (the host's double cos), NPOIN-point Gauss-Legendre
 * weights and abscissas on [-1, 1]; nothing written for npoin < 1. OK, BAD_SHAPE, KERNEL (a
 * root whose Newton iteration does not converge in 1000 steps; the Fortran's has no limit).
 * ww_snl1_gqm_f1f1f1: F1F1F1 on the host, the f1/f ratios of layout iq_om1 (1..7) into f1sf
 * (NF1+1 entries; layout 4 sets *nf1 = 40); returns the Fortran's message bits (0 when NF1 fits
 * the layout; 1, 2, 4, 8, 16 for layouts 1, 2, 3, 4, 7), or -BAD_SHAPE for a null pointer.
 * Status of all three in ww_snl1_gqm_last_error(). */
int ww_snl1_gqm_couple(int n, const double* k, double* coef, int* diag);
int ww_snl1_gqm_gauleg(int npoin, double* w_leg, double* x_leg);
int ww_snl1_gqm_f1f1f1(int* nf1, int iq_om1, double* f1sf);
int ww_snl1_gqm_last_error(void);

/* B200 extension. Selects the DIA kernel of grid `igrid`: 0 automatic (the pair kernel when
 * INSNL1's tables have the row-shift form and fit it, else the band kernel, else the row-shift
 * kernel, else the gather kernel; measured fastest in that order at 36x36 on B200), 1 the gather kernel over the
 * index tables, 2 the row-shift kernel (one CTA per point), 3 the band kernel (register
 * windows over frequency bands, TMA-staged input), 4 the tile kernel (the band kernel compiled
 * for 36 or 24 directions, zero-padded rows, no clamps), 5 the pair kernel (the band kernel over
 * two points at once, the additions paired FADD2; for 36 directions its form with the band
 * shape fixed at compile time, unrolled rows and zero-padded matrices), 6 the pair kernel's
 * general form for any grid it fits.
 * Returns the previous choice, or -1 for an unknown grid or a choice its tables cannot run. */
int ww_snl1_select_kernel(int igrid, int which);

/* B200 extension (the autotuner; no counterpart in the reference). Times every DIA kernel that
 * grid igrid's tables can run on 16,384 synthetic points of its spectral grid with CUDA events
 * (median of three launches after a warm-up), selects the fastest for the grid and records the
 * choice (ww_autotune_report). Synchronous; allocates its test arrays for the call. Returns the
 * kernel chosen (as ww_snl1_select_kernel numbers them), or -1. */
int ww_snl1_autotune(int igrid);

/* B200 extension, a test of the failure path (no counterpart in the reference). With bytes > 0
 * (at most 1024), every CTA of grid igrid's pair kernels expects that many bytes more than its
 * first bulk copy brings, so its bounded wait (about a second) runs out: the CTA stops, the
 * launch completes with the DIA's status word set, and ww_snl1 returns ERR_KERNEL; nothing
 * faults, hangs or stays in flight, and the next call with bytes = 0 runs normally. */
int ww_snl1_test_stall(int igrid, int bytes);

/* B200 extension (the autotuner). The W3SRCE kernels' CTAs per SM, each count with the
 * shared-memory carveout that fits it (the rest of the SM's memory is L1), timed on a sample
 * of the caller's own points (arguments as ww_srce_batch takes them, host arrays, read only:
 * the sample runs on device copies): the fastest is kept for every later W3SRCE launch in the
 * process. Synchronous. Returns the CTAs per SM chosen, or -1. */
int ww_srce_autotune(int igrid, int it, int inflags24, int flogrd57, int flogrd58, float dtg,
                     int npts, const float* spec, const float* wn1, const float* cg1,
                     const float* pin, const float* psc, const float* whitecap,
                     const float* taubbl, const float* tauice);

/* B200 extension: the autotuner's choices so far as a JSON object, {"<choice> <shape>
 * <device>": {"choice": c, "ms": {"<candidate>": median ms, ...}}, ...}, written to buf (at
 * most len - 1 characters and a NUL). Returns the full length, or -1. */
int ww_autotune_report(char* buf, int len);

/* ---------------------------------------------------------------- the resident spectrum VA */
/* VA(NSPEC, 0:NSEALM) of grid igrid, kept in HBM beside the Fortran array (resident_c.hpp:1-42).
 * `va` is VA(1,0), nspec = SIZE(VA,1), nsealm = UBOUND(VA,2); the first call binds the grid to
 * them and later calls with another address or shape are BAD_SHAPE. Return WwKokkosStatus. */

/* Replaces ww_va_host_read (resident_c.hpp:46): before a host read of VA, copy d_va back when
 * the device holds the newer bits; state BOTH. */
int ww_va_host_read(int igrid, float* va, int nspec, int nsealm);

/* Replaces ww_va_host_write (resident_c.hpp:49): ww_va_host_read, then state HOST. */
int ww_va_host_write(int igrid, float* va, int nspec, int nsealm);

/* Replaces ww_va_host_read_cols (resident_c.hpp:58): with state DEVICE, copy back only the
 * columns cols[0..ncol) (0..nsealm, duplicates allowed), gathered on the device; state kept. */
int ww_va_host_read_cols(int igrid, float* va, int nspec, int nsealm, int ncol, const int* cols);

/* Replaces ww_va_host_wrote_cols (resident_c.hpp:69): after host statements wrote exactly the
 * columns cols, with state DEVICE or BOTH push those columns into d_va; state kept. */
int ww_va_host_wrote_cols(int igrid, float* va, int nspec, int nsealm, int ncol, const int* cols);

/* Replaces ww_va_host_update (resident_c.hpp:75): before a host statement whose only writes of
 * VA zero whole columns; binds or checks, no copy. */
int ww_va_host_update(int igrid, float* va, int nspec, int nsealm);

/* Replaces ww_va_device_zero_cols (resident_c.hpp:84-85): d_va(:, cols) = 0 when the device
 * copy is newer or equal; state kept. */
int ww_va_device_zero_cols(int igrid, float* va, int nspec, int nsealm, int ncol,
                           const int* cols);

/* Replaces ww_va_device (resident_c.hpp:89): before a launch reads d_va of a bound grid: HOST
 * -> one H2D copy, state BOTH; write = 1 then marks DEVICE. */
int ww_va_device(int igrid, int write);

/* Replaces ww_va_report (resident_c.hpp:92): copy counters to stderr (at exit under
 * WW_KOKKOS_VA_COUNT=1). */
void ww_va_report(void);

/* B200 extension: the device address of grid igrid's d_va (NULL before its first device
 * sync), so a caller can run its own device code on the resident spectrum. */
void* ww_va_device_ptr(int igrid);

/* B200 extension: the state of grid igrid's VA: 0 HOST, 1 DEVICE, 2 BOTH, -1 unbound. */
int ww_va_state(int igrid);

/* ---------------------------------------------------------------- PR3/UQ propagation */

/* Replaces ww_ktp3_batch (prop3_c.hpp:75-81): W3KTP3 NTIMES times on each of NPTS sea points,
 * one intra-spectral part of W3WAVE. rpar[3] = DMIN, CTMAX, FACHFA; ipar[7] = NK, NTH, NSPEC,
 * NK2, FLCTH, FLCK, FLCUR; sig, dsip (NK+2); ecos, esin, ec2, esc, es2, mapwn, mapwn2
 * (NSPEC+NTH); mapth2 ((NK+2)*NTH); cg, wn (NK+2, 0:NSEA); jsea, isea (npts, 1-based);
 * pscal (10, npts) = CTHG0S, MAX(DMIN,DW), DDDX, DDDY, CX, CY, DCXDX, DCXDY, DCYDX, DCYDY;
 * va (NSPEC, 0:NSEALM) with ncol = NSEALM+1, updated in place; cflthmax, cflkmax (NSEALM)
 * written at JSEA. Returns a WwKokkosStatus. */
int ww_ktp3_batch(const float* rpar, int nrpar, const int* ipar, int nipar, const float* sig,
                  const float* dsip, const float* ecos, const float* esin, const float* ec2,
                  const float* esc, const float* es2, const int* mapwn, const int* mapth2,
                  const int* mapwn2, int itstep, int ntimes, float facth, float fack, int nsea,
                  const float* cg, const float* wn, int npts, const int* jsea, const int* isea,
                  const float* pscal, int ncol, float* va, float* cflthmax, float* cflkmax);

/* Replaces ww_ktp3_batch_va (prop3_c.hpp:86-94): ww_ktp3_batch on the resident VA of grid
 * igrid (synced to the device first; state DEVICE afterwards); cflthmax/cflkmax stay host
 * arrays. */
int ww_ktp3_batch_va(int igrid, const float* rpar, int nrpar, const int* ipar, int nipar,
                     const float* sig, const float* dsip, const float* ecos, const float* esin,
                     const float* ec2, const float* esc, const float* es2, const int* mapwn,
                     const int* mapth2, const int* mapwn2, int itstep, int ntimes, float facth,
                     float fack, int nsea, const float* cg, const float* wn, int npts,
                     const int* jsea, const int* isea, const float* pscal, float* va, int nspec,
                     int nsealm, float* cflthmax, float* cflkmax);

/* Replaces ww_xyp3_batch (prop3_c.hpp:25-32): W3GATH, W3XYP3, W3SCAT for every component
 * ISPEC with on[ISPEC-1] /= 0 (W3WAVE's ISPEC loop, W3_SHRD). rpar[5] = DTCFL, DTH, XFR, WDCG,
 * WDTH; ipar[11] = NX, NY, NSEA, NK, NTH, NSPEC, ICLOSE, FLCX, FLCY, FLAGLL, FLCUR; imaps[8] =
 * NMX0, NMX1, NMX2, NMY0, NMY1, NMY2, NACT, NCENT; tscal[3] = DSEC21 of the day, of TBPI0 to
 * TIME, of TBPI0 to TBPIN; mapsf (NSEA,3); clats (0:NSEA); sig (0:NK+1); ecos, esin
 * (NSPEC+NTH); dpdx, dpdy, dqdx, dqdy, gsqrt (NY,NX); atrnx, atrny (NY*NX,-1:1); mapx2, mapy2,
 * mapaxy, maptrn (0/1), mapsta (NY*NX); mapcxy (NSEA); cg (0:NK+1, 0:NSEA); cx, cy (0:NSEA);
 * flbpi, nbi, isbpi (NBI), bbpi0, bbpin (NSPEC, 0:NBI); on (NSPEC); va (NSPEC, 0:NSEALM) with
 * ncol = NSEALM+1. The averaging's order-dependent sums are reproduced bit for bit (an ordered
 * gather per target cell). Tripole grids are UNSUPPORTED, as in the reference. */
int ww_xyp3_batch(const float* rpar, int nrpar, const int* ipar, int nipar, const int* imaps,
                  int nimaps, const float* tscal, int ntscal, float dtg, const int* mapsf,
                  const float* clats, const float* sig, const float* ecos, const float* esin,
                  const float* dpdx, const float* dpdy, const float* dqdx, const float* dqdy,
                  const float* gsqrt, const float* atrnx, const float* atrny, const int* mapx2,
                  const int* mapy2, const int* mapaxy, const int* mapcxy, const int* maptrn,
                  const int* mapsta, const float* cg, const float* cx, const float* cy,
                  int flbpi, int nbi, const int* isbpi, const float* bbpi0, const float* bbpin,
                  const int* on, int ncol, float* va);

/* Replaces ww_xyp3_batch_va (prop3_c.hpp:37-46): ww_xyp3_batch on the resident VA of grid
 * igrid (synced to the device first, state DEVICE afterwards). */
int ww_xyp3_batch_va(int igrid, const float* rpar, int nrpar, const int* ipar, int nipar,
                     const int* imaps, int nimaps, const float* tscal, int ntscal, float dtg,
                     const int* mapsf, const float* clats, const float* sig, const float* ecos,
                     const float* esin, const float* dpdx, const float* dpdy, const float* dqdx,
                     const float* dqdy, const float* gsqrt, const float* atrnx,
                     const float* atrny, const int* mapx2, const int* mapy2, const int* mapaxy,
                     const int* mapcxy, const int* maptrn, const int* mapsta, const float* cg,
                     const float* cx, const float* cy, int flbpi, int nbi, const int* isbpi,
                     const float* bbpi0, const float* bbpin, const int* on, float* va, int nspec,
                     int nsealm);

/* Replaces ww_xyp3_batch_mpi (prop3_c.hpp:48-63, prop3_shim.cpp:1068-1099): ww_xyp3_batch_va
 * under W3_MPI. Sea point ISEA is column K = (ISEA-1)/naproc + 1 of rank IP =
 * MOD(ISEA-1,naproc) + 1. This rank's (iaproc's) points are its VA columns; rank IP's value of
 * the L-th component with on /= 0 (ascending) is rbuf[poff[IP-1] + L*nsealm + K-1] (W3GATH's
 * GSTORE), and W3SCAT writes the same place of sbuf (SSTORE, 0 past NSEA). poff holds the
 * blocks in rank order, NSPLOC*nsealm each (iaproc's entry not read); nbuf =
 * (naproc-1)*NSPLOC*nsealm. Other shapes: BAD_SHAPE, nothing written. */
int ww_xyp3_batch_mpi(int igrid, const float* rpar, int nrpar, const int* ipar, int nipar,
                      const int* imaps, int nimaps, const float* tscal, int ntscal, float dtg,
                      const int* mapsf, const float* clats, const float* sig, const float* ecos,
                      const float* esin, const float* dpdx, const float* dpdy, const float* dqdx,
                      const float* dqdy, const float* gsqrt, const float* atrnx,
                      const float* atrny, const int* mapx2, const int* mapy2, const int* mapaxy,
                      const int* mapcxy, const int* maptrn, const int* mapsta, const float* cg,
                      const float* cx, const float* cy, int flbpi, int nbi, const int* isbpi,
                      const float* bbpi0, const float* bbpin, const int* on, float* va,
                      int nspec, int nsealm, int naproc, int iaproc, const int* poff,
                      const float* rbuf, float* sbuf, int nbuf);

/* Replace ww_xyp3_mpi_pack / ww_xyp3_mpi_unpack (prop3_c.hpp:65-70, prop3_shim.cpp:1101-1123):
 * buf[J*nsealm + K-1] = VA(isps[J], K), K = 1 .. nsealm, from the resident VA of grid igrid
 * (pack: state unchanged), or back into it (unpack: state DEVICE afterwards). */
int ww_xyp3_mpi_pack(int igrid, float* va, int nspec, int nsealm, const int* isps, int nisp,
                     float* buf);
int ww_xyp3_mpi_unpack(int igrid, float* va, int nspec, int nsealm, const int* isps, int nisp,
                       const float* buf);

/* B200 extension; the reference has no C entry for it (its W3MAP3 runs inside the W3WAVE port
 * as one serial thread, prop_map3.hpp:100-340). W3MAP3 on the device, as ordered stream
 * compactions with the reference's results: mapsta (NY*NX) and mapsf (NSEA,3) in; mapx2,
 * mapy2, mapaxy (NY*NX), mapcxy (NSEA) and counts[8] = NMX0, NMX1, NMX2, NMY0, NMY1, NMY2,
 * NACT, NCENT out when gtype < 3 (GTYPE >= 3 leaves them); mapth2 ((NK+2)*NTH) and mapwn2
 * (NSPEC+NTH) written only when mapth2[0] is 0. List entries past the counters keep their
 * values. MAPSF must address cells of the grid (else BAD_SHAPE). */
int ww_map3(int nx, int ny, int nsea, int nk, int nth, int gtype, const int* mapsta,
            const int* mapsf, int* mapx2, int* mapy2, int* mapaxy, int* mapcxy, int* mapth2,
            int* mapwn2, int* counts);

/* ww_map3 on device arrays, on the caller's CUDA stream; counts (host, 8 ints) after a sync.
 * MAPSF is not checked (it is device memory). */
int ww_map3_device(int nx, int ny, int nsea, int nk, int nth, int gtype, const int* mapsta,
                   const int* mapsf, int* mapx2, int* mapy2, int* mapaxy, int* mapcxy,
                   int* mapth2, int* mapwn2, int* counts, void* stream);

/* B200 extension (prop_mapt.hpp:55-79): W3MAPT, MAPTRN (NY*NX, 0/1) of the NSEA sea cells from
 * ATRNX/ATRNY (NY*NX, -1:1); other cells keep their values. */
int ww_mapt(int nx, int ny, int nsea, const int* mapsf, const float* atrnx, const float* atrny,
            int* maptrn);

/* B200 extension (updt_utrn.hpp:93-362, W3UTRN of w3updtmd.F90:2809-3194): the transparencies
 * ATRNX/ATRNY (NY*NX, -1:1) from TRNX/TRNY (NY*NX), the ice concentration ICE (0:NSEA) and the
 * icebergs BERG (NSEA) of grid (NX, NY) with NSEA sea points (MAPSF (NSEA,3), MAPSTA (NY,NX),
 * HPFAC/HQFAC (NY,NX)). trny_before is the REAL just before TRNY(1) in the caller's memory
 * (read as TRNY(0) for a sea point in cell 1 under TRFLAG 1, 3, 5). The ice arrays may be null
 * when TRFLAG < 3. */
int ww_utrn(int nx, int ny, int nsea, int trflag, float fice0, float ficen, float ficel,
            float ffacberg, int flagll, float trny_before, const float* trnx, const float* trny,
            const int* mapsf, const int* mapsta, const float* hpfac, const float* hqfac,
            const float* ice, const float* berg, float* atrnx, float* atrny);

/* ---------------------------------------------------------------- a whole step as one graph */
/* B200 extension; the reference has no counterpart (its W3WAVE port calls the entries one by
 * one, wave_w3wave.hpp:577-800). Between ww_step_begin(igrid) and ww_step_end(igrid), the calls
 * ww_ktp3_batch_va, ww_xyp3_batch_va and ww_srce_batch_va of grid igrid are validated and their
 * inputs copied to device buffers the step owns, but their kernels do not run: they are
 * recorded, in call order. ww_step_end captures them into one CUDA graph; ww_step_run replays
 * it nrep times on the resident VA (state DEVICE afterwards) on `stream` (NULL: the library's
 * stream, synchronised before returning), with no host work and no copies besides one upload of
 * the VA when the host holds the newer copy (after ww_va_host_write). Each replay repeats
 * the recorded calls with their recorded scalars (the time of day, the boundary times, DTG);
 * W3SRCE's per-point packets (PSC, WHITECAP, TAUBBL, TAUICE, SHAVE) and W3KTP3's CFL maxima stay
 * on the device, the packets carrying over from one replay to the next. ww_xyp3_batch_mpi is not
 * recorded (UNSUPPORTED). Return WwKokkosStatus. */
int ww_step_begin(int igrid);
int ww_step_end(int igrid);
int ww_step_run(int igrid, int nrep, void* stream);
int ww_step_free(int igrid);
/* B200 extension: the recorded steps of ngrids distinct grids replayed nrep times, the grids one
 * after another in list order on `stream` (NULL: the library's stream, synchronised before
 * returning): several regional grids of uneven size on one GPU in one call, with no host work
 * besides the graph launches. Return WwKokkosStatus. */
int ww_steps_run(const int* igrids, int ngrids, int nrep, void* stream);
/* B200 extension: merges the recorded steps of ngrids distinct grids (each with exactly one
 * ww_srce_batch_va call, all with the same spectral grid and ST4 tables) into one graph: every
 * grid's calls before its W3SRCE batch, then ONE persistent W3SRCE launch over all the grids'
 * points with a single work queue, then the calls after. ww_steps_run with the same list (same
 * order) replays it instead of the grids' graphs one after another; recording or freeing a
 * member grid's step drops it, as does ngrids == 0. Return WwKokkosStatus. */
int ww_steps_fuse(const int* igrids, int ngrids);
/* The number of calls the grid's step holds, or -1 for a grid without one. */
int ww_step_ops(int igrid);
/* The number of nodes (kernels, memsets) of the grid's captured step graph, or -1. */
int ww_step_nodes(int igrid);

/* B200 extension: the status of the most recent ww_ktp3_* / ww_xyp3_* / ww_map3* / ww_mapt /
 * ww_utrn call (the reference returns it only). */
int ww_prop3_last_error(void);

/* ---------------------------------------------------------------- W3WAVE's support routines */
/* Replace the entries of ww_kokkos_c.hpp:893-921 (argument tables in the reference's
 * wave_support_shim.cpp): W3GATH, W3SCAT (W3_SHRD), W3UWND (WNT1, RWND), W3UTRN (IC0), W3DZXY,
 * W3MAP3, W3MAPT (PR3) and DISTAB. No per-grid state: every call passes its sizes, copies its
 * arrays in and its results out. Each returns OK, NOT_INITIALISED, BAD_SHAPE, KERNEL or RUNTIME
 * (BAD_SHAPE also for a MAPSF or MAPFS entry outside the grid, which the kernels would index).
 * MAPSF is MAPSF(MSEA,3); VA is VA(NSPEC, 0:NSEALM) with ncol = NSEALM+1 columns; FIELD is
 * FIELD(1-NY:NY*(NX+2)). WW_KOKKOS_WAVE_COUNT=1 prints "ww_kokkos: W3<R> calls: N" at exit. */
int ww_wave_gath(int ispec, int nspec, int nsea, int ncol, int msea, int nx, int ny,
                 const float* va, const int* mapsf, float* field);
int ww_wave_scat(int ispec, int nspec, int nsea, int ncol, int msea, int nx, int ny,
                 const int* mapsta, const float* field, const int* mapsf, float* va);
/* dt0n = DSEC21(TW0,TWN), dt0t = DSEC21(TW0,TIME) as stored REALs; wx0..dtn (NX,NY); cx, cy and
 * ua0..u10d (NSEA); UA0..ASI are written when flfrst, read otherwise. */
int ww_wave_uwnd(int flfrst, float dt0n, float dt0t, int flcur, float rwindc, int nsea, int msea,
                 int nx, int ny, const int* mapsf, const float* wx0, const float* wy0,
                 const float* dt0, const float* wxn, const float* wyn, const float* dtn,
                 const float* cx, const float* cy, float* ua0, float* uai, float* ud0,
                 float* udi, float* as0, float* asi, float* ua, float* ud, float* as,
                 float* u10, float* u10d);
/* trny[-1] is read as the Fortran's TRNY(0) under TRFLAG 1, 3, 5 when cell 1 is a sea point. */
int ww_wave_utrn(int nx, int ny, int nsea, int msea, int trflag, float fice0, float ficen,
                 float ficel, float ffacberg, int flagll, const float* trnx, const float* trny,
                 const int* mapsf, const int* mapsta, const float* hpfac, const float* hqfac,
                 const float* ice, const float* berg, float* atrnx, float* atrny);
int ww_wave_dzxy(int nsea, int nx, int ny, const float* zz, const int* mapsta, const int* mapfs,
                 const float* dpdx, const float* dpdy, const float* dqdx, const float* dqdy,
                 int flagll, int iclose, float* dzzdx, float* dzzdy);
/* GTYPE < 3 only (BAD_SHAPE otherwise); counts = NMX0..NMX2, NMY0..NMY2, NACT, NCENT. */
int ww_wave_map3(int nx, int ny, int nsea, int msea, int nk, int nth, int gtype, const int* mapsta,
                 const int* mapsf, int* mapx2, int* mapy2, int* mapaxy, int* mapcxy, int* mapth2,
                 int* mapwn2, int* counts);
int ww_wave_mapt(int nsea, int msea, int ncell, const int* mapsf, const float* atrnx,
                 const float* atrny, int* maptrn);
/* NAR1D must be 121; ewn1, ecg1 (0:NAR1D) in: the Fortran's tables (the differing values are
 * counted on stderr), out: the device's; n1max, dsie likewise. */
int ww_wave_distab(int nar1d, float* ewn1, float* ecg1, int* n1max, float* dsie);
/* W3CFLXY (w3pro3md.F90:1980-2136; the reference's device form prop_cflxy.hpp:61-135, which its
 * W3WAVE driver calls for JSEA = 1..NSEAL when FLOGRD(9,3), wave_w3wave.hpp:548-574; the
 * reference exports no C entry for it). cflxymax[ISEA-1] = CFLXYMAX(ISEA), ISEA = 1..NSEA: the
 * largest spatial CFL number over every (IK, ITH), with the compiled loop's MAX operand order.
 * mapsf (MSEA,3), columns 1-2 read; clats (0:NSEA); ecos, esin (NTH); dpdx..dqdy (NY,NX); cg
 * (0:NK+1, 0:NSEA); cx, cy (0:NSEA), read when flcur (may be NULL otherwise); mgp 0/1: the W3_MGP
 * form (VGX, VGY subtracted; the reference's driver uses 0). While grid igrid (> 0) records a step
 * (ww_step_begin) the call is recorded and CFLXYMAX of the replays stays on the device, as
 * ww_ktp3_batch_va's CFLTHMAX does; igrid 0 runs at once. */
int ww_wave_cflxy(int igrid, int nsea, int msea, int nx, int ny, int nk, int nth, int flcur,
                  int mgp, float dtg, float vgx, float vgy, const int* mapsf, const float* clats,
                  const float* ecos, const float* esin, const float* dpdx, const float* dpdy,
                  const float* dqdx, const float* dqdy, const float* cg, const float* cx,
                  const float* cy, float* cflxymax);

/* ---------------------------------------------------------------- gridded output (W3OUTG) */
/* Replaces ww_outg_va (outg_c.hpp:97-120): W3OUTG (VA, .FALSE., FLOUTG, FLOUTG2) of
 * w3iogomd.F90:1201-2380, sections 1-4 and the space-time extremes, on the resident VA of grid
 * igrid (read on the device; VA crosses only when the host holds the newer bits). ipar is the
 * WwOutgIpar packet (25 ints: NK, NTH, NSEAL, NSEA, NX, NY, NFLD, NOGRP, NGRPP, FLOUTG, FLOUTG2,
 * OARST, OMPG, P2MSF(2:3), E3DF(2,1:5), E3DF(3,1:5)), rpar the WwOutgRpar packet (10 reals: DTH,
 * XFR, FTE, FTWL, FTTR, UNDEF, STEXU, STEYU, STEDU, WSCUT). flogrd, flogr2, flogrr are LOGICAL(4)
 * (NOGRP,NGRPP); va is VA(1,0), nspec = SIZE(VA,1), nsealm = UBOUND(VA,2); cg, wn (0:NK+1,0:NSEA),
 * dw (0:NSEA), sig (0:NK+1), dden, dsii (NK), ecos .. esc (NTH), mapsf (NSEA,3), mapsta (NY,NX).
 * fields: the 46 arrays of WwOutgField (40 of NFLD; EF .. STH2M (NFLD, E3DF(2,k):E3DF(3,k)),
 * P2SMS (NFLD, P2MSF(2):P2MSF(3)); a 2-D field the grid does not allocate is NULL). The fields
 * are computed into device buffers kept between calls; those W3IOGO writes (FLOGRD under FLOUTG,
 * FLOGR2 under FLOUTG2) and, when OARST, those W3IORS writes (FLOGRR) come back, the others keep
 * their host bits. OK, NOT_INITIALISED, BAD_SHAPE, UNSUPPORTED (CALC_U3STOKES, SKEWNESS or
 * CALC_WBT requested: FLOLOC(6,8), (6,12), (8,7..9), (2,17); or the grid is recording a step),
 * a resident-VA status, RUNTIME, KERNEL. */
int ww_outg_va(int igrid, const int* ipar, int nipar, const float* rpar, int nrpar,
               const int* flogrd, const int* flogr2, const int* flogrr, float* va, int nspec,
               int nsealm, const float* cg, const float* wn, const float* dw, const float* sig,
               const float* dden, const float* dsii, const float* ecos, const float* esin,
               const float* ec2, const float* es2, const float* esc, const int* mapsf,
               const int* mapsta, float* const* fields, int nfields);

/* B200 extension: ww_outg_va on device arrays, launched on `stream` (a cudaStream_t; NULL the
 * legacy default stream) with no copy and no synchronisation. The packets and flogrd/flogr2 are
 * host memory and are checked as ww_outg_va checks them; d_va is VA(1,0) on the device; cg ..
 * mapsta as ww_outg_va, in device memory (a MAPSF cell outside the grid reads as land); ebd is
 * NK*NSEAL floats of device work; fields the 46 device arrays (every 1-D one; a 2-D one only
 * when requested). CGE keeps its values at points that are not sea. Status also in
 * ww_outg_last_error(). */
int ww_outg_device(const int* ipar, int nipar, const float* rpar, int nrpar, const int* flogrd,
                   const int* flogr2, const float* d_va, int nspec, int nsealm, const float* cg,
                   const float* wn, const float* dw, const float* sig, const float* dden,
                   const float* dsii, const float* ecos, const float* esin, const float* ec2,
                   const float* es2, const float* esc, const int* mapsf, const int* mapsta,
                   float* ebd, float* const* fields, int nfields, void* stream);

/* Replaces ww_outg_part (outg_c.hpp:122-125): section 6 of W3OUTG (w3iogomd.F90:2242-2340), the
 * partition fields from W3CPRT's table. ipar is the WwOutgPartIpar packet (13 ints: NSEAL, NSEA,
 * NX, NY, NROW, NOSWLL, NICP, NDTP, DIMP = 15, NOGRP, NGRPP, FLOUTG, FLOUTG2), rpar (UNDEF,
 * WSCUT); icprt (NICP,2), dtprt (DIMP,NDTP); fields the 17 arrays of WwOutgPartField (15 of
 * (NROW, 0:NOSWLL), PWST and PNR (NROW)). Field k comes back when FLOGRD(4,k) (FLOUTG) or
 * FLOGR2(4,k) (FLOUTG2) is set. OK, NOT_INITIALISED, BAD_SHAPE (also when a sea point's ICPRT
 * names columns outside DTPRT), RUNTIME, KERNEL. */
int ww_outg_part(const int* ipar, int nipar, const float* rpar, int nrpar, const int* flogrd,
                 const int* flogr2, const int* mapsf, const int* mapsta, const int* icprt,
                 const float* dtprt, float* const* fields, int nfields);

/* B200 extension: the status of the most recent ww_outg_va / ww_outg_part call. */
int ww_outg_last_error(void);

/* ---------------------------------------------------------------- ST4 source terms (W3SRC4MD) */
/* A grid is configured as the reference's (ww_kokkos_c.hpp:136-203): ww_st4_init with the
 * RPAR/IPAR packets (st4_params.hpp:79-154 layout: 84 reals, 9 ints), one ww_st4_set_real/int per
 * array (ArrayId of st4_arrays.hpp:41-61, with its rank, LBOUND and SHAPE as the Fortran has them;
 * copied, not borrowed), then ww_st4_commit, which checks every array the configuration needs and
 * copies them to the device. TAUT, TAUHFT, TAUHFT2, FWTABLE and the DEL* scalars are one copy per
 * process, the last registration wins. Point entries take npts points, every per-point scalar an
 * array of npts; OUT arguments are copied in as well as out; status in ww_st4_last_error().
 * WW_KOKKOS_ST4_TABLES=1: ww_st4_commit rebuilds the grid's and the module's tables with INSIN4 on
 * the device (the reference does it with its host C++, st4_shim.cpp:301-345), prints how many
 * values differ from the registered ones and uses the rebuilt ones. */

/* Replaces ww_st4_init (ww_kokkos_c.hpp:158). OK, NOT_INITIALISED, BAD_SHAPE, UNSUPPORTED (W3_FLX5,
 * or NTH > 128). */
int ww_st4_init(int igrid, const float* rpar, int nrpar, const int* ipar, int nipar);

/* Replace ww_st4_set_real / ww_st4_set_int (ww_kokkos_c.hpp:163-166). OK, NOT_INITIALISED, TABLE. */
int ww_st4_set_real(int igrid, int id, const float* data, int rank, const int* lbound,
                    const int* extent);
int ww_st4_set_int(int igrid, int id, const int* data, int rank, const int* lbound,
                   const int* extent);

/* Replaces ww_st4_commit (ww_kokkos_c.hpp:172). OK, NOT_INITIALISED, TABLE, RUNTIME. */
int ww_st4_commit(int igrid);

/* INSIN4(FLTABS) (w3src4md.F90:1014-1288 with TABU_STRESS, TABU_TAUHF, TABU_TAUHF2; the
 * reference's host C++ st4_insin4.cpp:96-264, st4_tabu_*.cpp, which it runs under
 * WW_KOKKOS_ST4_TABLES) on the device, bit for bit, for the packet rpar/ipar (ww_st4_init's) and
 * SIG, DSIP (0:MK+1), TH (MTH), ECOS (MSPEC+MTH). Outputs, column-major, each may be NULL:
 * satweights, satindices (2*(MTH/2-1)+1, MTH); iktab (MK, 2000); dcki, qbi (2000, 1300); cumulw
 * (MSPEC, MSPEC); taut (201, 201), tauhft (101, 201) when SINTAILPAR(1) > 0.5 and fltabs;
 * tauhft2 (101, 201, 51) when also TTAUWSHELTER > 0; del[5] = DELUST, DELALP, DELTAUW, DELU,
 * DELTAIL (the packet's values where INSIN4 sets none). OK, NOT_INITIALISED, BAD_SHAPE, KERNEL,
 * RUNTIME. */
int ww_st4_tables(const float* rpar, int nrpar, const int* ipar, int nipar, const float* sig,
                  const float* dsip, const float* th, const float* ecos, int fltabs,
                  float* satweights, int* satindices, int* iktab, float* dcki, float* qbi,
                  float* cumulw, float* taut, float* tauhft, float* tauhft2, float* del);

/* Replaces ww_sds4 (ww_kokkos_c.hpp:177): W3SDS4. a, srhs, ddiag, brlambda (nspec, npts);
 * k, cg (nk, npts); whitecap (4, npts); the scalars (npts). */
void ww_sds4(int igrid, int npts, const float* a, const float* k, const float* cg,
             const float* ustar, const float* usdir, const float* depth, const float* dair,
             const float* dlwmean, int flogrd57, int flogrd58, float* srhs, float* ddiag,
             float* brlambda, float* whitecap);

/* Replaces ww_sin4 (ww_kokkos_c.hpp:185): W3SIN4. a, k, s, d, llws (nspec, npts); cg (nk, npts). */
void ww_sin4(int igrid, int npts, const float* a, const float* cg, const float* k,
             const float* u, const float* ustar, const float* drat, const float* as,
             const float* usdir, const float* z0, const float* cd, float* tauwx, float* tauwy,
             float* tauwnx, float* tauwny, float* s, float* d, int* llws);

/* Replaces ww_spr4 (ww_kokkos_c.hpp:193): W3SPR4 with CALC_USTAR. a, llws (nspec, npts); cg, wn
 * (nk, npts); ustar, usdir INOUT. */
void ww_spr4(int igrid, int npts, const float* a, const float* cg, const float* wn,
             const float* u, const float* udir, const float* tauwx, const float* tauwy,
             const int* llws, float* ustar, float* usdir, float* emean, float* fmean,
             float* fmean1, float* wnmean, float* amax, float* cd, float* z0, float* charn,
             float* fmeanws, float* dlwmean);

/* Replaces ww_st4_enabled (ww_kokkos_c.hpp:198): 1 WW_KOKKOS_SDS4, 2 WW_KOKKOS_SIN4,
 * 3 WW_KOKKOS_SPR4, 4 WW_KOKKOS_ST4_TABLES. */
int ww_st4_enabled(int which);

/* Replaces ww_st4_last_error (ww_kokkos_c.hpp:201). */
int ww_st4_last_error(void);

/* ----------------------------------------------------------- W3SRCE (source-term integration) */
/* Replaces ww_srce_init (ww_kokkos_c.hpp:216): rpar (29), ipar (12) at srce_params.hpp:36-84's
 * indices; sig, dden (NK), ecos, esin, mapwn (NSPEC), copied. Needs ww_snl1_init and
 * ww_st4_commit of the grid. OK, NOT_INITIALISED, BAD_SHAPE, UNSUPPORTED (not switch_lab_shrd's
 * source terms; W3FLD2; DIA tables not in the row-shift form). */
int ww_srce_init(int igrid, const float* rpar, int nrpar, const int* ipar, int nipar,
                 const float* sig, const float* dden, const float* ecos, const float* esin,
                 const int* mapwn);

/* Replaces ww_srce (ww_kokkos_c.hpp:227): W3SRCE(srce_direct, ...) for one point, the arguments in
 * the order of the Fortran dummy list (spec (nspec), whitecap (4), taubbl (2), tauice (2) and
 * every pointer scalar INOUT). */
void ww_srce(int igrid, int it, int inflags24, int flogrd57, int flogrd58, float* spec,
             const float* wn1, const float* cg1, float d_inp, float u10abs, float u10dir,
             float as, float ice, float dtg, float dair, float coef, float* ustar,
             float* ustdir, float* tauwx, float* tauwy, float* dtdyn, float* fcut,
             float* tauox, float* tauoy, float* tauwix, float* tauwiy, float* tauwnx,
             float* tauwny, float* phiaw, float* charn, float* tws, float* phioc,
             float* whitecap, float* phibbl, float* taubbl, float* tauice, float* phice,
             float* tauocx, float* tauocy, float* wnmean, float* fpi, int* shave);

/* Replaces ww_srce_batch (ww_kokkos_c.hpp:266): W3SRCE for npts points of a time step. spec
 * (nspec, npts), psc (22, npts), whitecap (4, npts), taubbl, tauice (2, npts) INOUT; wn1, cg1
 * (nk, npts), pin (7, npts) IN; shave (npts) OUT. Packet rows as WwSrceBatchIn / WwSrceBatchScal
 * (ww_kokkos_c.hpp:231-251). One launch on a persistent grid with a work queue. */
void ww_srce_batch(int igrid, int it, int inflags24, int flogrd57, int flogrd58, float dtg,
                   int npts, float* spec, const float* wn1, const float* cg1, const float* pin,
                   float* psc, float* whitecap, float* taubbl, float* tauice, int* shave);

/* Replaces ww_srce_batch_va (resident_c.hpp:98): ww_srce_batch on the resident VA of the grid,
 * point k being VA(:, jsea[k]) (1 <= jsea[k] <= nsealm); the spectra are not copied. */
void ww_srce_batch_va(int igrid, int it, int inflags24, int flogrd57, int flogrd58, float dtg,
                      float* va, int nspec, int nsealm, int npts, const int* jsea,
                      const float* wn1, const float* cg1, const float* pin, float* psc,
                      float* whitecap, float* taubbl, float* tauice, int* shave);

/* B200 extension. ww_srce_batch on device-resident arrays (same shapes), launched on the CUDA
 * stream `stream` without copies or synchronisation; status in ww_srce_last_error(), execution
 * errors surface at the caller's next synchronisation. Calls of one grid on different streams
 * must not overlap (they share the grid's work-queue counter). */
void ww_srce_batch_device(int igrid, int it, int inflags24, int flogrd57, int flogrd58,
                          float dtg, int npts, float* spec, const float* wn1, const float* cg1,
                          const float* pin, float* psc, float* whitecap, float* taubbl,
                          float* tauice, int* shave, void* stream);

/* Replaces ww_srce_enabled (ww_kokkos_c.hpp:272): 1 if WW_KOKKOS_SRCE resolves to on. */
int ww_srce_enabled(void);

/* Replaces ww_srce_last_error (ww_kokkos_c.hpp:275). */
int ww_srce_last_error(void);

/* ---------------------------------------------------------------- run-time flags */

/* Replace ww_kokkos_flag / preset_status / strict / fallback_slot / fallback_add
 * (ww_kokkos_c.hpp:875-891, kokkos/src/fortran_iface/part_flags.cpp:67-135): a part's flag
 * WW_KOKKOS_<PART> = "1" is on (1), any other value off; unset, WW_KOKKOS_PRESET=<name> turns on
 * the parts of that preset (1), then WW_KOKKOS_ALL=1 turns on every part that is not opt-in (2).
 * ww_kokkos_preset_status: 0 no preset, 1 known, -1 unknown name. ww_kokkos_strict: 1 when
 * WW_KOKKOS_STRICT=1. The fallback slots count calls a caller left on the Fortran and print
 * the counts once at exit. */
int ww_kokkos_flag(const char* name);
int ww_kokkos_preset_status(void);
int ww_kokkos_strict(void);
int ww_kokkos_fallback_slot(const char* part);
void ww_kokkos_fallback_add(int slot);

/* ---------------------------------------------------------------- learned DIA surrogate */
/* B200 extensions with no counterpart in the reference (ww3-gpu has no learned component). The
 * surrogate stands in for W3SNL1 (snl1_team.hpp:351-497) behind a per-point gate; rejected
 * points are computed by the plain, bit-exact DIA kernel. Device pointers throughout, except
 * where an argument says host. Status codes as above, read with ww_mlp_last_error /
 * ww_sur_last_error. */

/* A plain MLP din -> dh -> dh -> dh -> dout with GELU (tanh form) between layers, BF16 weights
 * and activations, FP32 accumulation on the tensor cores (tcgen05) and FP32 master weights,
 * trained with AdamW. Widths are multiples of 64; the loss is the mean squared error over the
 * first nvalid output columns; cap is the largest training batch (a multiple of 128). */
int ww_mlp_create(int din, int dh, int dout, int nvalid, int cap, unsigned long long seed,
                  int* handle);
int ww_mlp_destroy(int handle);
/* Parameters as host floats, layer by layer: W (n x k, row-major) then b (n). */
long long ww_mlp_param_count(int handle);
int ww_mlp_set_params(int handle, const float* host);
int ww_mlp_get_params(int handle, float* host);
/* The gradient of the last ww_mlp_train_step with apply == 0, same layout. */
int ww_mlp_get_grads(int handle, float* host);
/* One step on `rows` rows (a multiple of 128): x bf16 (rows x din), t fp32 (rows x ldt).
 * Forward, loss, backward; with apply != 0 also an AdamW update (lr, decoupled decay wd).
 * loss3 (host, may be null) receives the step's loss. */
int ww_mlp_train_step(int handle, int rows, const void* x, const float* t, int ldt, float lr,
                      float wd, int apply, float* loss3);
/* Inference: out fp32 (rows x dout) from x bf16 (rows x din). */
int ww_mlp_forward(int handle, int rows, const void* x, float* out);
/* The library's tensor-core GEMM on its own: C = A . B^T with A bf16 (M x K, row stride lda),
 * B bf16 (N x K, row stride ldb), tile width bn (64, 128, 192, 256; N a multiple), K a multiple
 * of 64, and epilogue `mode`: 1 z = C + bias -> aux = z, out = gelu(z), out_t = out^T; 2 out =
 * gelu(C + bias); 3 out_f32 = C + bias; 4 out = C * gelu'(aux), out_t = out^T; 5 out_f32 += C
 * with the reduction split in `splits` parts. Mode 2 or 3 plus 16: the same on paired tiles (two
 * CTAs of a cluster per 256-row tile, tcgen05.mma.cta_group::2, each CTA holding half of B's
 * tile), the form the surrogate's inference uses. Synchronous on `stream`. */
int ww_mlp_gemm(int mode, int M, int N, int K, int bn, int splits, const void* a, int lda,
                const void* b, int ldb, const float* bias, void* out, void* out_t, void* aux,
                float* out_f32, int ldo, int ldt, void* stream);
int ww_mlp_last_error(void);

/* The surrogate of DIA grid igrid (ww_snl1_init first): an MLP with NSPEC + 2 inputs (the
 * log-normalised spectrum, rotated to its dominant direction, and two depth features), three
 * hidden layers of `nhidden`, NSPEC outputs (the normalised S_nl) and one error head. */
int ww_sur_init(int igrid, int nhidden, unsigned long long seed);
/* npts synthetic sea states (JONSWAP wind sea, cos^2s spreading, a swell system on a fraction
 * `bimodal` of points, depth log-uniform in [dmin, dmax]) as A (nspec x npts), CG (nk x npts),
 * KDMEAN (npts), seeded per point index p0 + i. */
int ww_sur_synth(int igrid, int npts, unsigned long long seed, float bimodal, float dmin,
                 float dmax, long long p0, float* a, float* cg, float* kdmean, void* stream);
/* Builds the training set on the device: npts synthetic sea states labelled by the plain DIA
 * kernel and normalised; the last `holdout` are never drawn by training. */
int ww_sur_dataset(int igrid, long long npts, long long holdout, unsigned long long seed,
                   float bimodal, float dmin, float dmax);
/* Weights of the loss terms besides the MSE: mu for the squared Hs-tendency error relative to
 * the gross tendency, lambda for the error head. */
int ww_sur_loss_weights(int igrid, float mu, float lambda);
/* `steps` AdamW steps on random batches of `batch` rows (warm-up, cosine decay lr -> lr_end);
 * losses (host, 3 x steps, may be null) receives each step's loss terms. */
int ww_sur_train(int igrid, int steps, int batch, float lr, float lr_end, float wd,
                 unsigned long long seed, float* losses);
/* Loss terms (host loss3) of the current network on dataset rows [p0, p0 + npts). */
int ww_sur_eval(int igrid, long long p0, int npts, float* loss3);
/* Gate thresholds: energy residual bound and predicted log-error bound. */
int ww_sur_gate(int igrid, float energy, float log_err);
/* Sets the gate from npts fresh synthetic points judged by the FP64 DIA: points whose energy
 * residual is within `energy` are accepted in order of predicted error while the mean Hs-
 * tendency error over all npts (a rejected point counting zero) stays within target_err.
 * out (host, 4): log-error threshold, accepted fraction, mean error with the gate, without. */
int ww_sur_calibrate(int igrid, int npts, unsigned long long seed, float bimodal, float dmin,
                     float dmax, float energy, float target_err, float* out);
/* The gated W3SNL1: arguments as ww_snl1_device (ww_kokkos_c.hpp:102-118 for their meaning),
 * plus accepted (npts ints, may be null): 1 where the surrogate's S was kept (D is then 0: the
 * surrogate does not model the diagonal term), 0 where the plain DIA computed S and D.
 * Asynchronous on `stream`. */
void ww_snl1_gated(int igrid, int npts, const float* a, const float* cg, const float* kdmean,
                   float* s, float* d, int* accepted, void* stream);
/* The gated W3SNL1 on host arrays, as ww_snl1 (ww_kokkos_c.hpp:115-116) takes them: the
 * copies in and out are pipelined with the compute in chunks of 65,536 points on three slots
 * (page-locked caller memory copies fastest); D is 0 where the surrogate was kept. Only S and
 * the rejected points' D rows cross the bus: host threads clear D while the device works (a
 * chunk rejecting more than 8,192 points brings its whole D). Synchronous. Status in
 * ww_sur_last_error(). */
void ww_snl1_gated_host(int igrid, int npts, const float* a, const float* cg,
                        const float* kdmean, float* s, float* d);
/* The network alone: out fp32 (rows x the padded output width, NSPEC + 1 rounded up to 64)
 * from normalised inputs x bf16 (rows x the padded input width, NSPEC + 2 rounded up to 64):
 * the four tensor-core GEMMs of one inference, asynchronous on `stream`. */
int ww_sur_forward(int igrid, int rows, const void* x, float* out, void* stream);
/* Points the last ww_snl1_gated sent to the plain DIA (synchronises `stream`), or -1. */
int ww_sur_fallback_count(int igrid, void* stream);
/* The FP64 DIA on npts points and the error of s_cand (may be null) against it: stats (npts x
 * 10 doubles, device) per point: Hs, Hs tendency of the FP64 S and of the candidate, gross Hs
 * tendency, band tendency error and magnitude, squared S error and FP64 S norm, mean-frequency
 * tendency of the FP64 S and of the candidate. s64, d64 (npts x nspec doubles) may be null. */
int ww_sur_judge(int igrid, int npts, const float* a, const float* cg, const float* kdmean,
                 const float* s_cand, double* stats, double* s64, double* d64, void* stream);
/* Trained state as host floats: the MLP's parameters (ww_mlp_set_params layout) then the NK
 * target scales. */
long long ww_sur_param_count(int igrid);
int ww_sur_get_params(int igrid, float* host);
int ww_sur_set_params(int igrid, const float* host);
int ww_sur_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* WW_B200_H */
