/* oracle/dia_body.h -- TEST INFRASTRUCTURE ONLY (included twice by oracle/dia_oracle.c).
 *
 * The DIA restated in plain C, once per working precision: R is the real type, F(name) the
 * libm function of that type (expf/exp ...), S(name) the suffixed symbol. Only tests, the
 * bench's CPU-baseline leg and smoke() call it, as the checker of the CUDA library.
 *
 * Followed reference code (ww3-gpu, paths within that project):
 *   INSNL1 -> kokkos/src/ww_kokkos/snl1_tables.cpp:82-329 (sections 1-9 of w3snl1md.F90 INSNL1)
 *   W3SNL1 -> kokkos/src/ww_kokkos/snl1_team.hpp:351-497 (sections 1-4 of w3snl1md.F90 W3SNL1)
 * Every expression keeps the reference's operand order; this file must be compiled with
 * -ffp-contract=off so no multiply-add is fused. */

/* Fortran x**n for a runtime integer n: the binary-exponent chain of libgcc's __powisf2
 * (snl1_tables.cpp:35-43). */
static R S(powi)(R x, int n) {
  unsigned m = (n < 0) ? (unsigned)(-n) : (unsigned)n;
  R y = (m & 1u) ? x : (R)1;
  while ((m >>= 1u) != 0u) {
    x = x * x;
    if (m & 1u) y = y * x;
  }
  return (n < 0) ? (R)1 / y : y;
}

/* x**11 by GCC's power tree at -O3: x^5 * x^6 (snl1_tables.cpp:53-59). */
static R S(pow11)(R x) {
  const R x2 = x * x;
  const R x3 = x2 * x;
  const R x5 = x2 * x3;
  const R x6 = x3 * x3;
  return x5 * x6;
}

typedef struct {
  int nfr, nfrhgh, nfrchg, nspecx, nspecy, nspec, nth;
  R dal1, dal2, dal3, awg[8], swg[8];
  int *ipim; /* 16 x nspecx: ip11..ip14, im11..im14, ip21..ip24, im21..im24 (0-based) */
  int *ic;   /* 16 x nspec : ic11, ic21 .. ic81, ic12, ic22 .. ic82 (0-based) */
  R *af11;   /* nspecx */
} S(tables);

static void S(tables_free)(S(tables) *t) {
  free(t->ipim);
  free(t->ic);
  free(t->af11);
  t->ipim = t->ic = NULL;
  t->af11 = NULL;
}

/* INSNL1. Returns 0, or -1 when the configuration is not usable. `o0_chain` selects how
 * AF11 = x**11 is multiplied out: 0 the power tree of a gfortran -O3 build of WW3 (the
 * reference's choice, snl1_tables.cpp:45-59), 1 libgcc's __powisf2 binary chain x^3 * x^8 of
 * a -O0 build (the one the reference's frozen golden vector was made with: the reference's
 * docs/log/2026-10-14-snl1-bitwise-af11.md). */
static int S(insnl1)(const oracle_snl1_config *c, const R *sig, int o0_chain, S(tables) *t) {
  const int nth = c->nth, nspec = c->nk * c->nth;
  const R one = (R)1, lam = (R)c->lam, dth = (R)c->dth, xfr = (R)c->xfr;
  memset(t, 0, sizeof *t);
  if (c->nk <= 0 || nth <= 0) return -1;
  t->nfr = c->nk;
  t->nth = nth;
  t->nspec = nspec;

  /* 1. Internal angles of the quadruplet. */
  const R lamm2_b = one - lam, lamp2_b = one + lam;
  const R lamm2 = lamm2_b * lamm2_b, lamp2 = lamp2_b * lamp2_b;
  const R delth3 = F(acos)((lamm2 * lamm2 + (R)4 - lamp2 * lamp2) / ((R)4 * lamm2));
  const R delth4 = F(asin)(-F(sin)(delth3) * lamm2 / lamp2);

  /* 2. Lambda-dependent weights. */
  const R p2 = lamp2_b * lamp2_b, m2 = lamm2_b * lamm2_b;
  t->dal1 = one / (p2 * p2);
  t->dal2 = one / (m2 * m2);
  t->dal3 = (R)2 * t->dal1 * t->dal2;

  /* 3. Directional indices (INT truncates toward zero). */
  const R cthp = F(fabs)(delth4 / dth);
  const int ithp = (int)cthp, ithp1 = ithp + 1;
  const R wthp = cthp - (R)ithp, wthp1 = one - wthp;
  const R cthm = F(fabs)(delth3 / dth);
  const int ithm = (int)cthm, ithm1 = ithm + 1;
  const R wthm = cthm - (R)ithm, wthm1 = one - wthm;

  /* 4. Frequency indices. */
  const R xfrln = F(log)(xfr);
  const int ifrp = (int)(F(log)(one + lam) / xfrln), ifrp1 = ifrp + 1;
  const R wfrp = (one + lam - S(powi)(xfr, ifrp)) / (S(powi)(xfr, ifrp1) - S(powi)(xfr, ifrp));
  const R wfrp1 = one - wfrp;
  const int ifrm = (int)(F(log)(one - lam) / xfrln), ifrm1 = ifrm - 1;
  const R wfrm = (S(powi)(xfr, ifrm) - (one - lam)) / (S(powi)(xfr, ifrm) - S(powi)(xfr, ifrm1));
  const R wfrm1 = one - wfrm;

  /* 5. Range of the extended spectrum. */
  t->nfrhgh = t->nfr + ifrp1 - ifrm1;
  t->nfrchg = t->nfr - ifrm1;
  t->nspecy = t->nfrhgh * nth;
  t->nspecx = t->nfrchg * nth;
  if (t->nfrchg <= 0) return -1;

  /* 7. Spectral addresses: IFn(IFR) row maps and ITn(ITH) wrapped direction shifts. */
  int *ifn = (int *)malloc(sizeof(int) * 8 * (size_t)t->nfrchg);
  int *itn = (int *)malloc(sizeof(int) * 8 * (size_t)nth);
  for (int ifr = 1; ifr <= t->nfrchg; ++ifr) {
    int *f = ifn + (size_t)(ifr - 1) * 8;
    f[0] = ifr + ifrp;
    f[1] = ifr + ifrp1;
    f[2] = ifr + ifrm > 0 ? ifr + ifrm : 0;
    f[3] = ifr + ifrm1 > 0 ? ifr + ifrm1 : 0;
    f[4] = ifr - ifrp > 0 ? ifr - ifrp : 0;
    f[5] = ifr - ifrp1 > 0 ? ifr - ifrp1 : 0;
    f[6] = ifr - ifrm;
    f[7] = ifr - ifrm1;
  }
  for (int ith = 1; ith <= nth; ++ith) {
    int *q = itn + (size_t)(ith - 1) * 8;
    q[0] = ith + ithp;
    q[1] = ith + ithp1;
    q[2] = ith + ithm;
    q[3] = ith + ithm1;
    q[4] = ith - ithp;
    q[5] = ith - ithp1;
    q[6] = ith - ithm;
    q[7] = ith - ithm1;
    for (int n = 0; n < 4; ++n) if (q[n] > nth) q[n] -= nth;
    for (int n = 4; n < 8; ++n) if (q[n] < 1) q[n] += nth;
  }
  /* address of (ITn, IFn) for bin (ith, ifr), all 1-based, stored minus one */
#define ADDR(IT, IF, ITH, IFR) \
  (itn[(size_t)((ITH)-1) * 8 + (IT)-1] + (ifn[(size_t)((IFR)-1) * 8 + (IF)-1] - 1) * nth - 1)
  /* (ITn, IFn) pairs of the tables, in the stored order (snl1_tables.cpp:186-223). */
  static const int kPm[16][2] = {{2, 2}, {1, 2}, {2, 1}, {1, 1}, {8, 4}, {7, 4}, {8, 3}, {7, 3},
                                 {6, 2}, {5, 2}, {6, 1}, {5, 1}, {4, 4}, {3, 4}, {4, 3}, {3, 3}};
  static const int kC[16][2] = {{6, 6}, {5, 6}, {6, 5}, {5, 5}, {4, 8}, {3, 8}, {4, 7}, {3, 7},
                                {2, 6}, {1, 6}, {2, 5}, {1, 5}, {8, 8}, {7, 8}, {8, 7}, {7, 7}};
  t->ipim = (int *)malloc(sizeof(int) * 16 * (size_t)t->nspecx);
  t->ic = (int *)malloc(sizeof(int) * 16 * (size_t)nspec);
  t->af11 = (R *)malloc(sizeof(R) * (size_t)t->nspecx);
  for (int isp = 0; isp < t->nspecx; ++isp) {
    const int ifr = 1 + isp / nth, ith = 1 + isp % nth;
    for (int j = 0; j < 16; ++j)
      t->ipim[(size_t)j * t->nspecx + isp] = ADDR(kPm[j][0], kPm[j][1], ith, ifr);
  }
  for (int isp = 0; isp < nspec; ++isp) {
    const int ifr = 1 + isp / nth, ith = 1 + isp % nth;
    for (int j = 0; j < 16; ++j)
      t->ic[(size_t)j * nspec + isp] = ADDR(kC[j][0], kC[j][1], ith, ifr);
  }
#undef ADDR
  free(ifn);
  free(itn);

  /* 8. The f**11 scaling array; beyond NK, FR grows by XFR each row. */
  const R tpiinv = (R)1 / ((R)2 * (R)(3.141592653589793));
  for (int ifr = 0; ifr < t->nfr; ++ifr) {
    const R v = o0_chain ? S(powi)(sig[ifr] * tpiinv, 11) : S(pow11)(sig[ifr] * tpiinv);
    for (int ith = 0; ith < nth; ++ith) t->af11[ith + ifr * nth] = v;
  }
  R fr = sig[t->nfr - 1] * tpiinv;
  for (int ifr = t->nfr; ifr < t->nfrchg; ++ifr) {
    fr = fr * xfr;
    const R v = o0_chain ? S(powi)(fr, 11) : S(pow11)(fr);
    for (int ith = 0; ith < nth; ++ith) t->af11[ith + ifr * nth] = v;
  }

  /* 9. Interpolation weights and their squares. */
  t->awg[0] = wthp * wfrp;
  t->awg[1] = wthp1 * wfrp;
  t->awg[2] = wthp * wfrp1;
  t->awg[3] = wthp1 * wfrp1;
  t->awg[4] = wthm * wfrm;
  t->awg[5] = wthm1 * wfrm;
  t->awg[6] = wthm * wfrm1;
  t->awg[7] = wthm1 * wfrm1;
  for (int j = 0; j < 8; ++j) t->swg[j] = t->awg[j] * t->awg[j];
  return 0;
}

/* W3SNL1 for one point with the index tables (gather form). `w` is scratch of
 * (NSPECY + NTH) + 8 * (NSPECX + NTH) + NSPEC values; a table entry j reads slot j + NTH. */
static void S(w3snl1_point)(const oracle_snl1_config *c, const S(tables) *t, const R *sig,
                            const R *a, const R *cg, R kdmean, R *s, R *d, R *w) {
  const int nth = t->nth, nfr = t->nfr, nspecx = t->nspecx, nspec = t->nspec;
  R *ue = w;
  R *arr[8];
  for (int k = 0; k < 8; ++k) arr[k] = ue + (t->nspecy + nth) + (size_t)k * (nspecx + nth);
  R *sa1 = arr[0], *sa2 = arr[1], *da1c = arr[2], *da1p = arr[3], *da1m = arr[4];
  R *da2c = arr[5], *da2p = arr[6], *da2m = arr[7];
  R *con = arr[7] + (nspecx + nth);
  const R dal1 = t->dal1, dal2 = t->dal2, dal3 = t->dal3;
  const R tpiinv = (R)1 / ((R)2 * (R)(3.141592653589793));

  /* 1. Proportionality constant (snl1_team.hpp:383-390); MAX(a,b) as (a < b) ? b : a. */
  const R x0 = (R)c->kdcon * kdmean;
  const R x = (x0 < (R)c->kdmn) ? (R)c->kdmn : x0;
  const R y0 = (R)c->snls3 * x;
  const R x2 = ((R)-1.e15 < y0) ? y0 : (R)-1.e15;
  const R cons = (R)c->snlc1 * ((R)1 + (R)c->snls1 / x * ((R)1 - (R)c->snls2 * x) * F(exp)(x2));

  /* 2. Auxiliary spectrum UE = A / CONX and the zero bins 1-NTH..0 (:392-413). */
  for (int ifr = 0; ifr < nfr; ++ifr) {
    const R conx = tpiinv / sig[ifr] * cg[ifr];
    for (int ith = 0; ith < nth; ++ith) {
      const int isp = ith + ifr * nth;
      ue[isp + nth] = a[isp] / conx;
      con[isp] = conx;
    }
  }
  for (int i = 0; i < nth; ++i) {
    ue[i] = 0;
    for (int k = 0; k < 8; ++k) arr[k][i] = 0;
  }
  /* Parametric tail, row by row upward (:419-426). */
  for (int ifr = nfr; ifr < t->nfrhgh; ++ifr)
    for (int ith = 0; ith < nth; ++ith) {
      const int isp = ith + ifr * nth;
      ue[isp + nth] = ue[isp] * (R)c->fachfe;
    }

  /* 3. Interactions over the extended spectrum (:433-473). */
#define T(j, isp) (t->ipim[(size_t)(j) * nspecx + (isp)] + nth)
  for (int isp = 0; isp < nspecx; ++isp) {
    const R e00 = ue[isp + nth];
    const R ep1 = t->awg[0] * ue[T(0, isp)] + t->awg[1] * ue[T(1, isp)] +
                  t->awg[2] * ue[T(2, isp)] + t->awg[3] * ue[T(3, isp)];
    const R em1 = t->awg[4] * ue[T(4, isp)] + t->awg[5] * ue[T(5, isp)] +
                  t->awg[6] * ue[T(6, isp)] + t->awg[7] * ue[T(7, isp)];
    const R ep2 = t->awg[0] * ue[T(8, isp)] + t->awg[1] * ue[T(9, isp)] +
                  t->awg[2] * ue[T(10, isp)] + t->awg[3] * ue[T(11, isp)];
    const R em2 = t->awg[4] * ue[T(12, isp)] + t->awg[5] * ue[T(13, isp)] +
                  t->awg[6] * ue[T(14, isp)] + t->awg[7] * ue[T(15, isp)];
    const R factor = cons * t->af11[isp] * e00;
    const R sa1a = e00 * (ep1 * dal1 + em1 * dal2);
    const R sa1b = sa1a - ep1 * em1 * dal3;
    const R sa2a = e00 * (ep2 * dal1 + em2 * dal2);
    const R sa2b = sa2a - ep2 * em2 * dal3;
    sa1[isp + nth] = factor * sa1b;
    sa2[isp + nth] = factor * sa2b;
    da1c[isp + nth] = cons * t->af11[isp] * (sa1a + sa1b);
    da1p[isp + nth] = factor * (dal1 * e00 - dal3 * em1);
    da1m[isp + nth] = factor * (dal2 * e00 - dal3 * ep1);
    da2c[isp + nth] = cons * t->af11[isp] * (sa2a + sa2b);
    da2p[isp + nth] = factor * (dal1 * e00 - dal3 * em2);
    da2m[isp + nth] = factor * (dal2 * e00 - dal3 * ep2);
  }
#undef T

  /* 4. Source and diagonal terms (:475-496); IC(j)1 is row j, IC(j)2 row 8+j. */
#define C1(j, isp) (t->ic[(size_t)(j) * nspec + (isp)] + nth)
#define C2(j, isp) (t->ic[(size_t)(8 + (j)) * nspec + (isp)] + nth)
  for (int isp = 0; isp < nspec; ++isp) {
    s[isp] = con[isp] * (-(R)2 * (sa1[isp + nth] + sa2[isp + nth]) +
                         t->awg[0] * (sa1[C1(0, isp)] + sa2[C2(0, isp)]) +
                         t->awg[1] * (sa1[C1(1, isp)] + sa2[C2(1, isp)]) +
                         t->awg[2] * (sa1[C1(2, isp)] + sa2[C2(2, isp)]) +
                         t->awg[3] * (sa1[C1(3, isp)] + sa2[C2(3, isp)]) +
                         t->awg[4] * (sa1[C1(4, isp)] + sa2[C2(4, isp)]) +
                         t->awg[5] * (sa1[C1(5, isp)] + sa2[C2(5, isp)]) +
                         t->awg[6] * (sa1[C1(6, isp)] + sa2[C2(6, isp)]) +
                         t->awg[7] * (sa1[C1(7, isp)] + sa2[C2(7, isp)]));
    d[isp] = -(R)2 * (da1c[isp + nth] + da2c[isp + nth]) +
             t->swg[0] * (da1p[C1(0, isp)] + da2p[C2(0, isp)]) +
             t->swg[1] * (da1p[C1(1, isp)] + da2p[C2(1, isp)]) +
             t->swg[2] * (da1p[C1(2, isp)] + da2p[C2(2, isp)]) +
             t->swg[3] * (da1p[C1(3, isp)] + da2p[C2(3, isp)]) +
             t->swg[4] * (da1m[C1(4, isp)] + da2m[C2(4, isp)]) +
             t->swg[5] * (da1m[C1(5, isp)] + da2m[C2(5, isp)]) +
             t->swg[6] * (da1m[C1(6, isp)] + da2m[C2(6, isp)]) +
             t->swg[7] * (da1m[C1(7, isp)] + da2m[C2(7, isp)]);
  }
#undef C1
#undef C2
}

/* The batch: a, s, d are (nspec, npts) and cg (nk, npts), column-major. */
static int S(w3snl1_batch)(const oracle_snl1_config *c, const R *sig, int npts, const R *a,
                           const R *cg, const R *kdmean, R *s, R *d, int nthreads,
                           int o0_chain) {
  S(tables) t;
  if (S(insnl1)(c, sig, o0_chain, &t) != 0) {
    S(tables_free)(&t);
    return -1;
  }
  const int nspec = t.nspec, nk = c->nk;
  const size_t wlen = (size_t)(t.nspecy + t.nth) + 8 * (size_t)(t.nspecx + t.nth) + (size_t)nspec;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    R *w = (R *)malloc(sizeof(R) * wlen);
#pragma omp for schedule(dynamic, 1)
    for (int ip = 0; ip < npts; ++ip)
      S(w3snl1_point)(c, &t, sig, a + (size_t)ip * nspec, cg + (size_t)ip * nk, kdmean[ip],
                      s + (size_t)ip * nspec, d + (size_t)ip * nspec, w);
    free(w);
  }
  S(tables_free)(&t);
  return 0;
}
