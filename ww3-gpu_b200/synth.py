"""Seeded synthetic sea states for the DIA: JONSWAP spectra with cos^2s spreading.

The reference measures W3SNL1 on WW3 sea states (its frozen fixture and WW3 regtests); no such
data travels here, so these seeded spectra stand in, with the shapes and distributions of the
36x36 workload: frequencies geometric from 0.0373 Hz with ratio 1.1, 10-degree directions,
Hs ~ U(0.5, 8) m, fp ~ U(0.06, 0.2) Hz, gamma ~ U(1, 5), spreading cos^2s((th - thm)/2) with
s ~ U(2, 20) and a random mean direction thm. Intermediates are float64, outputs float32.

Action density and mean relative depth follow the reference's DIA benchmark generator
(ww3-gpu bench/dia/bench_dia.F90:81-107): A = E(sigma, theta) * Cg / sigma, with k and Cg from
the linear dispersion relation (Newton on sigma^2 = g k tanh(k d)) and
Cg = sigma / k / 2 * (1 + 2kd / sinh(min(2kd, 80))); KDMEAN = sum(E k d) / sum(E).
"""

import numpy as np

GRAV = 9.806  # ww3-gpu kokkos/src/ww_kokkos/st4_params.hpp:28
TPI_F32 = np.float32(2.0) * np.float32(np.pi)


def spectral_grid(nk=36, nth=36, f1=0.0373, xfr=1.1):
    """SIG(1:NK) (rad/s, float32, each a factor XFR above the last) and DTH = TPI / NTH."""
    xfr32 = np.float32(xfr)
    sig = np.empty(nk, np.float32)
    sig[0] = np.float32(TPI_F32 * np.float32(f1))
    for k in range(1, nk):
        sig[k] = np.float32(sig[k - 1] * xfr32)
    dth = np.float32(TPI_F32 / np.float32(nth))
    return sig, dth


def dia_config(nk=36, nth=36, xfr=1.1, lam=0.25, c_nl=2.78e7, kdconv=0.75, kdmin=0.5,
               cs1=5.5, cs2=0.833, cs3=-1.25, fachf=5.0):
    """ww_snl1_init's scalars for the DIA constants of the workload (SNLC1 = C / g^4,
    FACHFE = XFR^-FACHF)."""
    sig, dth = spectral_grid(nk, nth, xfr=xfr)
    cfg = {
        "nk": nk, "nth": nth, "xfr": float(np.float32(xfr)), "dth": float(dth),
        "lam": float(np.float32(lam)), "snlc1": float(np.float32(c_nl / GRAV ** 4)),
        "kdcon": float(np.float32(kdconv)), "kdmn": float(np.float32(kdmin)),
        "snls1": float(np.float32(cs1)), "snls2": float(np.float32(cs2)),
        "snls3": float(np.float32(cs3)),
        "fachfe": float(np.float32(np.float32(xfr) ** np.float32(-fachf))),
    }
    return cfg, sig


def wavenumber(sig, depth, iters=30):
    """k(sigma, d) from sigma^2 = g k tanh(k d), Newton from the deep-water value; float64.
    sig (nk,), depth (npts,) -> k (npts, nk)."""
    s = np.asarray(sig, np.float64)[None, :]
    d = np.asarray(depth, np.float64)[:, None]
    k = np.broadcast_to(s * s / GRAV, (d.shape[0], s.shape[1])).copy()
    for _ in range(iters):
        kd = np.minimum(k * d, 40.0)
        t = np.tanh(kd)
        f = GRAV * k * t - s * s
        fp = GRAV * t + GRAV * k * d / np.cosh(kd) ** 2
        k = k - f / fp
    return k


def sea_states(npts, seed=0, nk=36, nth=36, depth=4000.0, depth_range=None, bimodal=0.0):
    """npts seeded JONSWAP points: returns dict(a (npts, nspec), cg (npts, nk), kdmean (npts,),
    depth (npts,), hs (npts,)) with float32 spectra. ``depth_range=(lo, hi)`` draws depths
    log-uniformly instead of the fixed ``depth``; ``bimodal`` is the fraction of points that get
    an added swell system."""
    rng = np.random.default_rng(seed)
    cfg, sig = dia_config(nk, nth)
    dth = np.float64(cfg["dth"])
    s64 = sig.astype(np.float64)
    f = s64 / (2 * np.pi)
    th = np.arange(nth) * dth
    xfr = np.float64(cfg["xfr"])
    dsii = 0.5 * s64 * (xfr - 1.0 / xfr)  # band widths in sigma

    hs = rng.uniform(0.5, 8.0, npts)
    fp = rng.uniform(0.06, 0.2, npts)
    gam = rng.uniform(1.0, 5.0, npts)
    spr = rng.uniform(2.0, 20.0, npts)
    thm = rng.uniform(0.0, 2 * np.pi, npts)
    if depth_range is None:
        dep = np.full(npts, float(depth))
    else:
        lo, hi = depth_range
        dep = np.exp(rng.uniform(np.log(lo), np.log(hi), npts))
    swell = rng.uniform(0, 1, npts) < bimodal
    hs_sw = rng.uniform(0.5, 3.0, npts)
    fp_sw = rng.uniform(0.05, 0.09, npts)
    thm_sw = rng.uniform(0.0, 2 * np.pi, npts)

    def jonswap(fpk, gk):
        ff = f[None, :]
        fpp = fpk[:, None]
        sg = np.where(ff <= fpp, 0.07, 0.09)
        r = np.exp(-((ff - fpp) ** 2) / (2.0 * sg * sg * fpp * fpp))
        return ff ** -5 * np.exp(-1.25 * (fpp / ff) ** 4) * gk[:, None] ** r

    def spreading(tm, sk):
        x = np.cos(0.5 * (th[None, :] - tm[:, None])) ** 2
        dd = x ** sk[:, None]
        return dd / (dd.sum(axis=1, keepdims=True) * dth)

    def energy(hsk, fpk, gk, tm, sk):
        ef = jonswap(fpk, gk) / (2 * np.pi)  # density in sigma
        e = ef[:, :, None] * spreading(tm, sk)[:, None, :]  # (npts, nk, nth)
        m0 = (e * dsii[None, :, None]).sum(axis=(1, 2)) * dth
        return e * ((hsk / 4.0) ** 2 / m0)[:, None, None]

    e = energy(hs, fp, gam, thm, spr)
    if swell.any():
        idx = np.nonzero(swell)[0]
        e[idx] += energy(hs_sw[idx], fp_sw[idx], np.full(idx.size, 3.3), thm_sw[idx],
                         np.full(idx.size, 20.0))
    k = wavenumber(sig, dep)
    kd = k * dep[:, None]
    cg = 0.5 * s64[None, :] / k * (1.0 + 2.0 * kd / np.sinh(np.minimum(2.0 * kd, 80.0)))
    a = e * (cg / s64[None, :])[:, :, None]
    esum = e.sum(axis=2)
    kdmean = (esum * kd).sum(axis=1) / np.maximum(esum.sum(axis=1), np.finfo(np.float64).tiny)
    m0 = (e * dsii[None, :, None]).sum(axis=(1, 2)) * dth
    return {
        "a": a.reshape(npts, nk * nth).astype(np.float32),
        "cg": cg.astype(np.float32),
        "kdmean": kdmean.astype(np.float32),
        "depth": dep.astype(np.float32),
        "hs": (4.0 * np.sqrt(m0)).astype(np.float32),
    }


def sea_states_chunked(npts, seed=0, chunk=32768, out=None, **kw):
    """sea_states for large npts, chunk by chunk (chunk j seeded seed*1_000_003 + j), written
    into ``out`` = dict of preallocated arrays when given."""
    nk, nth = kw.get("nk", 36), kw.get("nth", 36)
    if out is None:
        out = {"a": np.empty((npts, nk * nth), np.float32), "cg": np.empty((npts, nk), np.float32),
               "kdmean": np.empty(npts, np.float32)}
    for j, p0 in enumerate(range(0, npts, chunk)):
        n = min(chunk, npts - p0)
        g = sea_states(n, seed=seed * 1_000_003 + j, **kw)
        for key in out:
            out[key][p0:p0 + n] = g[key]
    return out


# ---------------------------------------------------------------------------- PR3/UQ inputs
def spectral_arrays(nk=36, nth=36, f1=0.0373, xfr=1.1):
    """W3GDATMD's spectral arrays for the PR3 entries, float32, built as WW3's W3GRID does:
    SIG(0:NK+1) and DSIP(0:NK+1) from SIGMA = FR1*TPI/XFR**2 grown by XFR each bin, DSIP =
    SIG*(XFR-1/XFR)/2; TH = (ITH-1)*DTH; ECOS, ESIN, EC2, ESC, ES2 and MAPWN over NSPEC+NTH
    (the last NTH entries repeat the first row's trig values, MAPWN = NK+1 there)."""
    nspec = nk * nth
    x = np.float32(xfr)
    sxfr = np.float32(0.5) * (x - np.float32(1.0) / x)
    sig = np.empty(nk + 2, np.float32)
    dsip = np.empty(nk + 2, np.float32)
    sigma = np.float32(np.float32(f1) * TPI_F32 / (x * x))
    for ik in range(nk + 2):
        sigma = np.float32(sigma * x)
        sig[ik] = sigma
        dsip[ik] = np.float32(sigma * sxfr)
    dth = np.float32(TPI_F32 / np.float32(nth))
    th = (np.arange(nth, dtype=np.float32) * dth).astype(np.float32)
    ecos = np.cos(th.astype(np.float64)).astype(np.float32)
    esin = np.sin(th.astype(np.float64)).astype(np.float32)
    ecos[np.abs(ecos) < 1e-5] = 0.0
    esin[np.abs(esin) < 1e-5] = 0.0
    ec = np.tile(ecos, nk + 1)
    es = np.tile(esin, nk + 1)
    mapwn = np.repeat(np.arange(1, nk + 2, dtype=np.int32), nth)
    return {"sig": sig, "dsip": dsip, "dth": float(dth), "ecos": ec, "esin": es,
            "ec2": (ec * ec).astype(np.float32), "esc": (ec * es).astype(np.float32),
            "es2": (es * es).astype(np.float32), "mapwn": mapwn, "nspec": nspec}


def prop3_spectral_maps(nk, nth):
    """MAPTH2 ((NK+2)*NTH) and MAPWN2 (NSPEC+NTH), W3MAP3 section 5 (the reference's
    kokkos/src/ww_kokkos/prop_map3.hpp:242-275): 1-based indices into the rotated (NK+2, NTH)
    work spectrum; MAPWN2 lists wavenumbers 1..NK-1, then the NK row, then the zero row."""
    nk2 = nk + 2
    mapth2 = np.zeros(nk2 * nth, np.int32)
    for ik in range(1, nk + 1):
        for ith in range(1, nth + 1):
            mapth2[(ith + (ik - 1) * nth) - 1] = (ik + 1) + (ith - 1) * nk2
    mapwn2 = []
    for ik in range(1, nk):
        for ith in range(1, nth + 1):
            mapwn2.append((ik + 1) + (ith - 1) * nk2)
    mapwn2 += [nk + 1 + (ith - 1) * nk2 for ith in range(1, nth + 1)]
    mapwn2 += [1 + (ith - 1) * nk2 for ith in range(1, nth + 1)]
    return mapth2, np.array(mapwn2, np.int32)


def ktp3_case(npts, seed=0, nk=36, nth=36, nsea=None, depth_range=(5.0, 4000.0), ntloc=2,
              dtg=900.0, currents=True, spectra="jonswap"):
    """Seeded inputs of ww_ktp3_batch for npts sea points of a grid with nsea points (points
    listed in a shuffled order, every other column of VA left untouched). Returns a dict with
    the C ABI's arguments by name (column-major arrays flattened as the ABI reads them).
    spectra="uniform" fills VA with U(0, 1) values instead of sea states (grids of 10^5-10^6
    points, where only the index arithmetic at size is under test)."""
    rng = np.random.default_rng(seed)
    nsea = nsea or npts
    nspec, nk2 = nk * nth, nk + 2
    sp = spectral_arrays(nk, nth)
    mapth2, mapwn2 = prop3_spectral_maps(nk, nth)
    dep = np.exp(rng.uniform(np.log(depth_range[0]), np.log(depth_range[1]), nsea + 1))
    k = wavenumber(sp["sig"], dep)  # (nsea+1, nk+2), column ISEA = row here
    kd = np.minimum(k * dep[:, None], 40.0)
    s64 = sp["sig"].astype(np.float64)[None, :]
    cg = 0.5 * s64 / k * (1.0 + 2.0 * kd / np.sinh(np.minimum(2.0 * kd, 80.0)))
    nsealm = nsea
    va = _spectra(spectra, nsea, seed + 17, nk, nth, depth_range)
    isea = rng.permutation(np.arange(1, nsea + 1))[:npts].astype(np.int32)
    jsea = isea.copy()  # one rank: JSEA = ISEA
    lat = rng.uniform(-70.0, 70.0, npts)
    dmin = np.float32(0.1)
    pscal = np.zeros((npts, 10), np.float32)
    pscal[:, 0] = -np.tan(np.deg2rad(lat)) / 6.3661975e6
    pscal[:, 1] = np.maximum(dmin, dep[isea])
    pscal[:, 2] = rng.normal(0.0, 2e-3, npts)
    pscal[:, 3] = rng.normal(0.0, 2e-3, npts)
    if currents:
        pscal[:, 4] = rng.normal(0.0, 0.3, npts)
        pscal[:, 5] = rng.normal(0.0, 0.3, npts)
        pscal[:, 6:10] = rng.normal(0.0, 2e-5, (npts, 4))
    dth = np.float32(sp["dth"])
    return {
        "rpar": np.array([dmin, 0.7, np.float32(1.1) ** np.float32(-7.0)], np.float32),
        "ipar": np.array([nk, nth, nspec, nk2, 1, 1, int(currents)], np.int32),
        "sig": sp["sig"], "dsip": sp["dsip"], "ecos": sp["ecos"], "esin": sp["esin"],
        "ec2": sp["ec2"], "esc": sp["esc"], "es2": sp["es2"], "mapwn": sp["mapwn"],
        "mapth2": mapth2, "mapwn2": mapwn2,
        "facth": float(np.float32(dtg / (float(dth) * ntloc))),
        "fack": float(np.float32(dtg / ntloc)), "nsea": nsea,
        "cg": cg.astype(np.float32).reshape(-1), "wn": k.astype(np.float32).reshape(-1),
        "npts": npts, "jsea": jsea, "isea": isea, "pscal": pscal.reshape(-1),
        "va": va, "nsealm": nsealm,
        "cflthmax": np.full(nsealm, -1.0, np.float32), "cflkmax": np.full(nsealm, -1.0, np.float32),
    }


def _spectra(kind, nsea, seed, nk, nth, depth_range):
    """VA(NSPEC, 0:NSEA) as a C-ordered (nsea + 1, nspec) array, column 0 zero: seeded sea
    states, or U(0, 1) values for kind "uniform"."""
    va = np.zeros((nsea + 1, nk * nth), np.float32)
    if kind == "uniform":
        va[1:] = np.random.default_rng(seed).random((nsea, nk * nth), dtype=np.float32)
    else:
        va[1:] = sea_states(nsea + 1, seed=seed, nk=nk, nth=nth, depth_range=depth_range)["a"][1:]
    return va


def land_mask(nx, ny, seed=0, sea_fraction=0.7, smooth=6):
    """Seeded smooth random land/sea mask (True = sea), periodic in longitude; the first and
    last latitude rows are land, as W3GRID requires of a grid with PR3 propagation."""
    rng = np.random.default_rng(seed)
    f = rng.standard_normal((ny, nx))
    k = np.exp(-0.5 * (np.arange(-3 * smooth, 3 * smooth + 1) / smooth) ** 2)
    # longitude: periodic padding (wraps as often as needed when NX is below the kernel)
    f = np.apply_along_axis(lambda r: np.convolve(np.pad(r, 3 * smooth, mode="wrap"), k, "valid"),
                            1, f)
    # latitude: edge-padded, so the mask keeps NY rows whatever NY is against the kernel
    f = np.apply_along_axis(lambda c: np.convolve(np.pad(c, 3 * smooth, mode="edge"), k, "valid"),
                            0, f)
    sea = f > np.quantile(f, 1.0 - sea_fraction)
    sea[0, :] = False
    sea[-1, :] = False
    return sea


def sea_grid(nx, ny, seed=0, sea_fraction=0.7, boundary=0.02, excluded=0.01):
    """A seeded NX x NY lon/lat grid's MAPSTA (1 active sea, 2 boundary input, -1 excluded sea,
    0 land; rows 1 and NY land) flattened column-major as MAPSTA(NY,NX), and MAPSF(NSEA,3) of
    its sea points numbered row by row (IY outer), as W3GRID numbers them."""
    rng = np.random.default_rng(seed + 101)
    sea = land_mask(nx, ny, seed=seed, sea_fraction=sea_fraction)
    sta = np.where(sea, 1, 0).astype(np.int32)  # (NY, NX)
    u = rng.uniform(0.0, 1.0, sta.shape)
    sta[sea & (u < boundary)] = 2
    sta[sea & (u >= boundary) & (u < boundary + excluded)] = -1
    iy, ix = np.nonzero(sta != 0)  # row-major over (IY, IX): IY outer, IX inner
    ix = (ix + 1).astype(np.int32)
    iy = (iy + 1).astype(np.int32)
    mapsf = np.concatenate([ix, iy, (ix - 1) * ny + iy]).astype(np.int32)
    mapsta = np.ascontiguousarray(sta.T).reshape(-1).astype(np.int32)
    return mapsta, mapsf, int(ix.size)


def xyp3_case(nx=48, ny=32, seed=0, nk=36, nth=36, iclose=2, flcur=True, flbpi=True,
              on_fraction=1.0, dtg=900.0, ref=None, spectra="jonswap", on_components=None):
    """Seeded inputs of ww_xyp3_batch on an NX x NY regular lon/lat grid (0.25 degrees), the
    W3MAP3 maps built by ``ref`` (a callable ref(nx, ny, nsea, nk, nth, mapsta, mapsf) returning
    (mapx2, mapy2, mapaxy, mapcxy, counts), the reference's own W3MAP3 in the tests).
    spectra="uniform" fills VA with U(0, 1) values (see ktp3_case); on_components=n switches on
    n spectral components spread evenly over NSPEC instead of a random on_fraction."""
    rng = np.random.default_rng(seed)
    nspec = nk * nth
    sea = land_mask(nx, ny, seed=seed)
    mapsta2 = np.where(sea, 1, 0).astype(np.int32)  # (NY, NX)
    # a few active boundary points and excluded sea points
    cand = np.argwhere(sea)
    pick = rng.permutation(len(cand))
    for j in pick[: max(1, len(cand) // 50)]:
        mapsta2[tuple(cand[j])] = 2
    for j in pick[max(1, len(cand) // 50): max(2, len(cand) // 50 + len(cand) // 100)]:
        mapsta2[tuple(cand[j])] = -1
    # sea points row by row (IY outer), IXY = (IX-1)*NY + IY
    ix_l, iy_l = [], []
    for iy in range(1, ny + 1):
        for ix in range(1, nx + 1):
            if mapsta2[iy - 1, ix - 1] != 0:
                ix_l.append(ix)
                iy_l.append(iy)
    nsea = len(ix_l)
    ix_a = np.array(ix_l, np.int32)
    iy_a = np.array(iy_l, np.int32)
    mapsf = np.concatenate([ix_a, iy_a, (ix_a - 1) * ny + iy_a]).astype(np.int32)
    mapsta = np.ascontiguousarray(mapsta2.T).reshape(-1).astype(np.int32)  # column-major (NY,NX)
    mapx2, mapy2, mapaxy, mapcxy, counts = ref(nx, ny, nsea, nk, nth, mapsta, mapsf)
    nxy = nx * ny
    sp = spectral_arrays(nk, nth)
    sx = sy = 0.25
    lat = -80.0 + (np.arange(1, ny + 1) - 0.5) * (160.0 / ny)
    clat_cell = np.cos(np.deg2rad(lat))
    clats = np.ones(nsea + 1, np.float32)
    clats[1:] = clat_cell[iy_a - 1]
    ones = np.ones(nxy, np.float32)
    dpdx = (ones / sx).astype(np.float32)
    dqdy = (ones / sy).astype(np.float32)
    dpdy = np.zeros(nxy, np.float32)
    dqdx = np.zeros(nxy, np.float32)
    gsqrt = np.repeat(clat_cell[None, :], nx, axis=0).reshape(-1).astype(np.float32) * sx * sy
    atrnx = np.ones((3, nxy), np.float32)
    atrny = np.ones((3, nxy), np.float32)
    tr = rng.uniform(0.0, 1.0, (3, nxy)) < 0.05
    atrnx[tr] = rng.uniform(0.2, 1.0, tr.sum())
    atrny[tr] = rng.uniform(0.2, 1.0, tr.sum())
    maptrn = (rng.uniform(0.0, 1.0, nxy) < 0.03).astype(np.int32)
    dep = np.exp(rng.uniform(np.log(10.0), np.log(4000.0), nsea + 1))
    k = wavenumber(sp["sig"], dep)
    kd = np.minimum(k * dep[:, None], 40.0)
    cg = 0.5 * sp["sig"].astype(np.float64)[None, :] / k * (
        1.0 + 2.0 * kd / np.sinh(np.minimum(2.0 * kd, 80.0)))
    cx = np.zeros(nsea + 1, np.float32)
    cy = np.zeros(nsea + 1, np.float32)
    if flcur:
        cx[1:] = rng.normal(0.0, 0.4, nsea)
        cy[1:] = rng.normal(0.0, 0.4, nsea)
    bnd = np.nonzero(mapsta2.T.reshape(-1)[(ix_a - 1) * ny + iy_a - 1] == 2)[0] + 1  # ISEA
    if flbpi and len(bnd) > 0:
        isbpi = np.concatenate([bnd, bnd[:1]]).astype(np.int32)  # one point listed twice
    else:
        isbpi = np.zeros(1, np.int32)
    nbi = len(isbpi) if flbpi else 0
    va = _spectra(spectra, nsea, seed + 5, nk, nth, (10.0, 4000.0))
    bb0 = np.zeros((max(nbi, 0) + 1, nspec), np.float32)
    bbn = np.zeros((max(nbi, 0) + 1, nspec), np.float32)
    if nbi:
        gb = sea_states(2 * nbi, seed=seed + 9, nk=nk, nth=nth)
        bb0[1:] = gb["a"][:nbi]
        bbn[1:] = gb["a"][nbi:]
    on = (rng.uniform(0.0, 1.0, nspec) < on_fraction).astype(np.int32)
    if on_components is not None:
        on = np.zeros(nspec, np.int32)
        on[np.linspace(0, nspec - 1, on_components).round().astype(int)] = 1
    return {
        "rpar": np.array([300.0, sp["dth"], 1.1, 1.5, 1.5], np.float32),
        "ipar": np.array([nx, ny, nsea, nk, nth, nspec, iclose, 1, 1, 1, int(flcur)], np.int32),
        "imaps": np.asarray(counts, np.int32),
        "tscal": np.array([3600.0, 450.0, 900.0], np.float32), "dtg": float(np.float32(dtg)),
        "mapsf": mapsf, "clats": clats, "sig": sp["sig"], "ecos": sp["ecos"], "esin": sp["esin"],
        "dpdx": dpdx, "dpdy": dpdy, "dqdx": dqdx, "dqdy": dqdy, "gsqrt": gsqrt,
        "atrnx": atrnx.reshape(-1), "atrny": atrny.reshape(-1), "mapx2": mapx2, "mapy2": mapy2,
        "mapaxy": mapaxy, "mapcxy": mapcxy, "maptrn": maptrn, "mapsta": mapsta,
        "cg": cg.astype(np.float32).reshape(-1), "cx": cx, "cy": cy, "flbpi": int(flbpi),
        "nbi": nbi, "isbpi": isbpi, "bbpi0": bb0.reshape(-1), "bbpin": bbn.reshape(-1),
        "on": on, "va": va, "nsea": nsea, "nx": nx, "ny": ny,
    }


# ------------------------------------------------------------------------ ST4 and W3SRCE inputs
# The ST4 / W3SRCE packets and grid arrays of a synthetic WW3 grid. WW3's namelist defaults are not
# part of the reference (it only names them); the values below are in the ranges of WW3's ST4
# (Ardhuin et al. 2010) configurations and exercise every branch the kernels translate: the
# saturation-based breaking (SSDSC(1) = 1) with a directional sector (SSDSDTH < 180), the default
# O(NK^2 NTH^2) cumulative term (SSDSC(3) < 0), swell damping through FWTABLE (SSWELLF(2) /= 0),
# the tabulated stress and tail (SINTAILPAR(1) > 0.5, TTAUWSHELTER > 0) and the whitecap
# outputs. Parity does not depend on the values: the oracle and the kernels get the same arrays.
ST4_NRPAR, ST4_NIPAR = 84, 9
SRCE_NRPAR, SRCE_NIPAR = 29, 12


def st4_setup(nk=36, nth=36, xfr=1.1, f1=0.0373, variant="default"):
    """ST4 rpar/ipar (float32/int32) and grid arrays (float32, at the Fortran lower bounds:
    sig = SIG(0:NK+1), dsip = DSIP(0:NK+1), dden = DDEN(1:NK), sig2, dden2 (NSPEC),
    esin, ecos (NSPEC+NTH), th (NTH), fwtable (0:300)). variant "analytic" uses the analytic
    tail and Newton friction velocity (SINTAILPAR(1) < 0.5), "romero" the SSDSC(1) = 3 breaking."""
    sig1, dth = spectral_grid(nk, nth, f1=f1, xfr=xfr)
    x = np.float32(xfr)
    sig = np.empty(nk + 2, np.float32)
    sig[1:nk + 1] = sig1
    sig[0] = np.float32(sig1[0] / x)
    sig[nk + 1] = np.float32(sig1[-1] * x)
    sigstep = np.float32(0.5) * (x - np.float32(1.0) / x)
    dsip = (sig * sigstep).astype(np.float32)
    dden = (np.float32(dth) * dsip[1:nk + 1] * sig1).astype(np.float32)
    nspec = nk * nth
    th = (np.arange(nth, dtype=np.float64) * float(dth)).astype(np.float32)
    mapwn = np.repeat(np.arange(1, nk + 1), nth)
    mapth = np.tile(np.arange(1, nth + 1), nk)
    sig2 = sig[mapwn].astype(np.float32)
    dden2 = dden[mapwn - 1].astype(np.float32)
    ec = np.cos(th.astype(np.float64)).astype(np.float32)
    es = np.sin(th.astype(np.float64)).astype(np.float32)
    ecos = np.concatenate([ec[mapth - 1], ec]).astype(np.float32)
    esin = np.concatenate([es[mapth - 1], es]).astype(np.float32)
    # FWTABLE(0:300): a smooth friction-factor curve over log10(a/z0) in [-1, 8] (DELAB = 0.03).
    delab = np.float32(9.0 / 300.0)
    xab = -1.0 + np.arange(301) * float(delab)
    fwtable = (0.24 * np.exp(-0.9 * np.maximum(xab, 0.0)) + 0.002).astype(np.float32)

    r = np.zeros(ST4_NRPAR, np.float32)
    R = {"DTH": 0, "XFR": 1, "FTE": 2, "FTF": 3, "AAIRCMIN": 4, "AAIRGB": 5, "IGPARS5": 6,
         "WWNMEANPTAIL": 7, "SSTXFTFTAIL": 8, "AALPHA": 9, "BBETA": 10, "ZZ0MAX": 11,
         "ZZ0RAT": 12, "ZZALP": 13, "SSINTHP": 14, "TTAUWSHELTER": 15, "SSWELLF": 16,
         "SSDSC": 23, "SSDSBR": 44, "SINTAILPAR": 45, "SSDSP": 50, "WWNMEANP": 51,
         "SSTXFTWN": 52, "SSDSBRF1": 53, "SSDSBINT": 54, "SSDSBCK": 55, "SSDSHCK": 56,
         "SSDSABK": 57, "SSDSPBK": 58, "CAPCHNK": 59, "ZZWND": 69, "SSDSCOS": 70,
         "SSDSDTH": 71, "SSDSBT": 72, "SSDSBM": 73, "DELUST": 78, "DELALP": 79, "DELTAUW": 80,
         "DELU": 81, "DELTAIL": 82, "DELAB": 83}
    assert R["DELAB"] + 1 == 84
    sn = float(sig1[-1])
    r[R["DTH"]] = dth
    r[R["XFR"]] = x
    r[R["FTE"]] = 0.25 * sn * float(dth) * sn
    r[R["FTF"]] = 0.20 * float(dth) * sn
    r[R["AAIRCMIN"]] = 2.0
    r[R["AAIRGB"]] = 0.2
    r[R["WWNMEANPTAIL"]] = -0.5
    r[R["SSTXFTFTAIL"]] = 0.25
    r[R["AALPHA"]] = 0.0095
    r[R["BBETA"]] = 1.52
    r[R["ZZ0MAX"]] = 0.0
    r[R["ZZ0RAT"]] = 0.04
    r[R["ZZALP"]] = 0.006
    r[R["SSINTHP"]] = 2.0
    r[R["TTAUWSHELTER"]] = 1.0
    r[R["SSWELLF"]:R["SSWELLF"] + 7] = [0.66, -0.018, 0.022, 1.5e5, 1.2, 0.0, 2.3e5]
    sdsc = np.zeros(21, np.float32)
    sdsc[0] = 1.0          # saturation-based breaking
    sdsc[1] = -2.2e-5      # SDSC2
    sdsc[2] = -0.40344     # SDSCUM < 0: the default cumulative branch
    sdsc[4] = 0.0
    sdsc[5] = 0.3          # isotropic part
    sdsc[6] = 0.3          # whitecap width
    sdsc[11] = 1.0         # SIG power of the mean direction weights
    sdsc[19] = 1.0
    r[R["SSDSC"]:R["SSDSC"] + 21] = sdsc
    r[R["SSDSBR"]] = 0.0009
    r[R["SINTAILPAR"]:R["SINTAILPAR"] + 5] = [1.0, 1.0, 0.0, 1.0, 0.11]
    r[R["SSDSP"]] = 2.0
    r[R["WWNMEANP"]] = 0.5
    r[R["SSTXFTWN"]] = 0.2
    r[R["SSDSBRF1"]] = 0.5
    r[R["ZZWND"]] = 10.0
    r[R["SSDSCOS"]] = 2.0
    r[R["SSDSDTH"]] = 80.0
    r[R["SSDSBT"]] = 0.0
    r[R["SSDSBM"]:R["SSDSBM"] + 5] = [0.0, 1.0, 0.0, 0.0, 0.0]
    r[R["DELAB"]] = delab
    if variant == "analytic":
        r[R["SINTAILPAR"]:R["SINTAILPAR"] + 5] = [0.0, 1.0, 0.0, 1.0, 0.11]
        r[R["TTAUWSHELTER"]] = 0.0
    if variant == "romero":
        sdsc3 = sdsc.copy()
        sdsc3[0] = 3.0
        sdsc3[1] = 5.0e-5
        sdsc3[8] = 0.05
        sdsc3[12] = 1.0
        sdsc3[13] = 1.0
        sdsc3[14] = 1.0
        sdsc3[15] = 1.2
        sdsc3[17] = 0.5
        sdsc3[18] = 1.0
        sdsc3[10] = 1.0
        sdsc3[7] = 1.0
        r[R["SSDSC"]:R["SSDSC"] + 21] = sdsc3
        r[R["SSDSBT"]] = 0.001
    ipar = np.array([nk, nth, nspec, nk, nth, nspec, 0, 0, 0], np.int32)
    return {"rpar": r, "ipar": ipar, "sig": sig, "sig2": sig2, "dsip": dsip, "dden": dden,
            "dden2": dden2, "esin": esin, "ecos": ecos, "th": th, "fwtable": fwtable,
            "mapwn": mapwn.astype(np.int32), "R": R, "nk": nk, "nth": nth, "dth": dth}


def srce_setup(st, ln1=0, seed=0):
    """W3SRCE rpar/ipar and grid arrays (SIG, DDEN (NK), ECOS, ESIN (NSPEC), MAPWN (NSPEC)) for
    the ST4 grid ``st`` of st4_setup. ``seed`` switches W3_SEED, ``ln1`` W3SLN1."""
    nk, nth = st["nk"], st["nth"]
    sig1 = st["sig"][1:nk + 1]
    x = float(st["rpar"][1])
    r = np.zeros(SRCE_NRPAR, np.float32)
    lnx = np.log(x)
    r[0] = 0.3                                   # DMIN
    r[1] = 300.0                                 # DTMAX
    r[2] = 15.0                                  # DTMIN
    r[3] = 1.0 / lnx                             # FACTI1
    r[4] = 1.0 - np.log(float(sig1[0])) / lnx    # FACTI2
    r[5] = x ** -7.0                             # FACHFA = XFR**(-FACHF-2)
    r[6] = 0.62e-3 * (2 * np.pi) ** 4 / GRAV ** 2  # FACP
    r[7] = 0.0                                   # XFLT
    r[8] = 0.1                                   # XREL
    r[9] = 0.8                                   # FHMAX
    r[10] = 2.5 * 2 * np.pi                      # FFXFM
    r[11] = 4.0 * GRAV / 28.0                    # FFXPM
    r[12] = 0.0                                  # FFXFA
    r[13:17] = 0.0                               # ICESCALES
    r[17] = 1.0e-6                               # SLNC1
    r[18] = 1.0                                  # FSPM
    r[19] = 1.0                                  # FSHF
    r[20] = -0.067 / GRAV                        # SBTC1
    r[21] = 0.25                                 # SDBC1
    r[22] = 0.8                                  # SDBC2
    r[23] = 0.9                                  # FACSD
    ipar = np.array([nk, nth, nk * nth, 1, 0, 0, 0, 1, ln1, seed, 0, 0], np.int32)
    return {"rpar": r, "ipar": ipar, "sig": sig1.copy(), "dden": st["dden"].copy(),
            "ecos": st["ecos"][:nk * nth].copy(), "esin": st["esin"][:nk * nth].copy(),
            "mapwn": st["mapwn"].copy()}


def srce_points(npts, seed=0, nk=36, nth=36, depth_range=(10.0, 4000.0)):
    """Per-point W3SRCE inputs: spec (npts, nspec) action density, wn1, cg1 (npts, nk), pin
    (npts, 7: D_INP U10ABS U10DIR AS ICE DAIR COEF), psc (npts, 22) and whitecap (npts, 4),
    taubbl, tauice (npts, 2). Winds U10 ~ U(3, 25) m/s from a random direction."""
    g = sea_states(npts, seed=seed, nk=nk, nth=nth, depth_range=depth_range)
    rng = np.random.default_rng(seed + 7)
    sig, _ = spectral_grid(nk, nth)
    k = wavenumber(sig, g["depth"])
    u10 = rng.uniform(3.0, 25.0, npts)
    udir = rng.uniform(0.0, 2 * np.pi, npts)
    pin = np.zeros((npts, 7), np.float32)
    pin[:, 0] = g["depth"]
    pin[:, 1] = u10
    pin[:, 2] = udir
    pin[:, 5] = 1.225
    pin[:, 6] = 1.0
    psc = np.zeros((npts, 22), np.float32)
    psc[:, 0] = 0.035 * u10          # USTAR
    psc[:, 1] = udir                 # USTDIR
    psc[:, 2] = 0.5 * (0.035 * u10) ** 2 * np.cos(udir)  # TAUWX
    psc[:, 3] = 0.5 * (0.035 * u10) ** 2 * np.sin(udir)
    return {"spec": g["a"], "wn1": k.astype(np.float32), "cg1": g["cg"], "pin": pin,
            "psc": psc, "whitecap": np.zeros((npts, 4), np.float32),
            "taubbl": np.zeros((npts, 2), np.float32), "tauice": np.zeros((npts, 2), np.float32)}


def st4_tables_own(st):
    """The ST4 tables of ``st`` that the analytic-tail configuration reads, built here (not by
    the reference), for inputs of runs that have no reference at hand: SATINDICES/SATWEIGHTS
    and CUMULW by INSIN4's formulas (w3src4md.F90:1134-1153, :1252-1282: weights
    cos(th_i - th_j)**SSDSCOS over +-SDSNTH directions; the distance
    sqrt(c^2 + c2^2 - 2 c c2 cos(dth)) * DSIP(ik2) / (c2 / 2) * DTH of deep-water phase speeds
    c = g / sigma for IK2 <= IK - DIKCUMUL), DCKI/QBI/IKTAB zero (INSIN4 fills them only for
    SSDSBCK > 0), no stress tables (SINTAILPAR(1) < 0.5). Same dict layout as the oracle's."""
    ipar, r, R = st["ipar"], st["rpar"], st["R"]
    nk, nth, nspec, mk, mth, mspec = [int(v) for v in ipar[:6]]
    assert float(r[R["SINTAILPAR"]]) < 0.5, "own tables cover the analytic tail only"
    dth = np.float32(r[R["DTH"]])
    rade = np.float32(180.0) / np.float32(np.pi)
    nsat = 2 * (mth // 2 - 1) + 1
    sati = np.ones((mth, nsat), np.int32)   # (ith, row), written Fortran-ordered below
    satw = np.zeros((mth, nsat), np.float32)
    th = st["th"].astype(np.float64)
    if float(r[R["SSDSDTH"]]) < 180.0:
        sdsnth = min(int(np.floor(float(r[R["SSDSDTH"]]) / float(dth * rade) + 0.5)), nth // 2 - 1)
        for ith in range(1, nth + 1):
            for i_int in range(ith - sdsnth, ith + sdsnth + 1):
                j = i_int + nth if i_int < 1 else (i_int - nth if i_int > nth else i_int)
                row = i_int - (ith - sdsnth) + 1
                sati[ith - 1, row - 1] = j
                satw[ith - 1, row - 1] = np.float32(
                    np.cos(th[ith - 1] - th[j - 1]) ** float(r[R["SSDSCOS"]]))
    else:
        satw[:] = 1.0
    cumulw = np.zeros((mspec, mspec), np.float32)  # (is, is2): C order of the Fortran (is2, is)
    if float(r[R["SSDSC"] + 2]) < 0:
        xfr = float(r[R["XFR"]])
        dik = int(np.floor(float(r[R["SSDSBRF1"]]) / (xfr - 1.0) + 0.5))
        sig = st["sig"].astype(np.float64)
        ec = st["ecos"].astype(np.float64)
        for ik in range(1, nk + 1):
            c = GRAV / sig[ik]
            for ik2 in range(1, ik - dik + 1):
                c2 = GRAV / sig[ik2]
                d = np.abs(np.arange(nth)[:, None] - np.arange(nth)[None, :])  # |ith2 - ith|
                v = np.sqrt(c * c + c2 * c2 - 2 * c * c2 * ec[d]) * float(st["dsip"][ik2]) / \
                    (0.5 * c2) * float(dth)
                cumulw[(ik - 1) * nth:ik * nth, (ik2 - 1) * nth:ik2 * nth] = v.T
    return {"satweights": satw.reshape(-1), "satindices": sati.reshape(-1),
            "iktab": np.zeros(mk * 2000, np.int32), "dcki": np.zeros(2000 * 1300, np.float32),
            "qbi": np.zeros(2000 * 1300, np.float32), "cumulw": cumulw.reshape(-1),
            "taut": None, "tauhft": None, "tauhft2": None, "rpar": r.copy(), "nsat": nsat}


def st4_registrations(st, t):
    """(id, array, is_int, lbounds, extents) of every ST4 array as ww_st4_set_real/int takes
    them: ArrayId, rank and LBOUND of the reference's table (st4_arrays.hpp:41-81)."""
    ipar = st["ipar"]
    nk, nth, nspec, mk, mth, mspec = [int(v) for v in ipar[:6]]
    nsat = t["nsat"]
    regs = [
        (0, st["sig"], False, [0], [nk + 2]), (1, st["sig2"], False, [1], [nspec]),
        (2, st["dsip"], False, [0], [nk + 2]), (3, st["dden"], False, [1], [nk]),
        (4, st["dden2"], False, [1], [nspec]), (5, st["esin"], False, [1], [nspec + nth]),
        (6, st["ecos"], False, [1], [nspec + nth]), (7, st["th"], False, [1], [nth]),
        (8, t["satweights"], False, [1, 1], [nsat, mth]),
        (9, t["cumulw"], False, [1, 1], [mspec, mspec]),
        (10, t["dcki"], False, [1, 1], [2000, 1300]), (11, t["qbi"], False, [1, 1], [2000, 1300]),
        (12, t["satindices"], True, [1, 1], [nsat, mth]),
        (13, t["iktab"], True, [1, 1], [mk, 2000]), (17, st["fwtable"], False, [0], [301]),
    ]
    if t.get("taut") is not None:
        regs.append((14, t["taut"], False, [0, 0], [201, 201]))
        regs.append((15, t["tauhft"], False, [0, 0], [101, 201]))
    if t.get("tauhft2") is not None:
        regs.append((16, t["tauhft2"], False, [0, 0, 0], [101, 201, 51]))
    return regs


# W3OUTG packets (outg_c.hpp:12-47, :74-104): FLOGRD(NOGRP, NGRPP) with WW3's NOGRP = 10 and
# NGRPP = 18, and the (group, index) entries the device W3OUTG leaves to the Fortran.
OUTG_NOGRP, OUTG_NGRPP = 10, 18
OUTG_UNSUPPORTED = ((6, 8), (6, 12), (8, 7), (8, 8), (8, 9), (2, 17))


def outg_flags(select="all", seed=0):
    """FLOGRD as int32 (NOGRP*NGRPP, column-major): every output the device W3OUTG computes
    ("all"), none ("none"), or a seeded half of them ("some")."""
    f = np.zeros(OUTG_NOGRP * OUTG_NGRPP, np.int32)
    if select == "none":
        return f
    rng = np.random.default_rng(seed + 17)
    for j in range(1, OUTG_NGRPP + 1):
        for i in range(1, OUTG_NOGRP + 1):
            if (i, j) in OUTG_UNSUPPORTED:
                continue
            f[(i - 1) + (j - 1) * OUTG_NOGRP] = 1 if select == "all" else int(rng.uniform() < 0.5)
    return f


def outg_case(nx=40, ny=30, seed=0, nk=30, nth=24, xfr=1.1, ompg=0, ste=(1000.0, 1000.0, 3600.0),
              select="all", floutg2=0, oarst=0, nsealm_extra=2, e3df=None, p2=(3, 12)):
    """Seeded inputs of ww_outg_va on an NX x NY grid (sea_grid: active, boundary and excluded
    points), JONSWAP spectra of random depth (some points calm: a zero spectrum), the W3GDATMD
    arrays at their Fortran bounds, FLOGRD/FLOGR2/FLOGRR, and 46 prefilled field arrays (EF ..
    STH2M over E3DF(2,k):E3DF(3,k), P2SMS over P2MSF(2):P2MSF(3)). ``ste`` = (STEXU, STEYU, STEDU);
    ``e3df`` = (E3DF(2,1:5), E3DF(3,1:5)) and ``p2`` = P2MSF(2:3) may reach outside 1..NK."""
    rng = np.random.default_rng(seed)
    mapsta, mapsf, nsea = sea_grid(nx, ny, seed=seed)
    nsealm = nsea + nsealm_extra
    sp = spectral_arrays(nk, nth, xfr=xfr)
    sig = sp["sig"]
    dth = np.float32(sp["dth"])
    x = np.float32(xfr)
    dsii = np.empty(nk, np.float32)
    dsii[:] = np.float32(0.5) * sig[1:nk + 1] * (x - np.float32(1.0) / x)
    dsii[0] = np.float32(0.5) * sig[1] * (x - np.float32(1.0))
    dsii[nk - 1] = np.float32(0.5) * sig[nk] * (x - np.float32(1.0)) / x
    dden = (dth * dsii * sig[1:nk + 1]).astype(np.float32)
    th = np.arange(nth, dtype=np.float64) * float(dth)
    ecos = np.cos(th).astype(np.float32)
    esin = np.sin(th).astype(np.float32)
    ecos[np.abs(ecos) < 1e-5] = 0.0
    esin[np.abs(esin) < 1e-5] = 0.0
    st = sea_states(nsea, seed=seed + 5, nk=nk, nth=nth, depth_range=(1.0, 3000.0), bimodal=0.3)
    va = np.zeros((nsealm + 1, nk * nth), np.float32)
    va[1:nsea + 1] = st["a"]
    calm = rng.uniform(0, 1, nsea) < 0.05
    va[1:nsea + 1][calm] = 0.0
    va[nsea + 1:] = rng.uniform(0, 1e-3, (nsealm - nsea, nk * nth)).astype(np.float32)
    dep = np.concatenate([[1.0], st["depth"].astype(np.float64)])
    s64 = sig.astype(np.float64)
    k = wavenumber(s64, dep)
    kd = k * dep[:, None]
    cg = 0.5 * s64[None, :] / k * (1.0 + 2.0 * kd / np.sinh(np.minimum(2.0 * kd, 80.0)))
    signk = sig[nk]
    fte = np.float32(0.25) * signk * dth * signk
    ftwl = np.float32(GRAV / 6.0) / (signk * signk) * dth * signk
    fttr = np.float32(0.20) * dth * signk
    rpar = np.array([dth, x, fte, ftwl, fttr, -999.9, ste[0], ste[1], ste[2], 0.8], np.float32)
    e3df2, e3df3 = e3df if e3df is not None else ([1, 3, 1, 2, 5], [nk, 10, nk, 20, nk - 1])
    ipar = np.array([nk, nth, nsea, nsea, nx, ny, nsealm, OUTG_NOGRP, OUTG_NGRPP, 1, floutg2,
                     oarst, ompg, p2[0], p2[1], *e3df2, *e3df3], np.int32)
    fields = [rng.standard_normal(nsealm).astype(np.float32) for _ in range(40)]
    for k3 in range(5):
        fields.append(rng.standard_normal((e3df3[k3] - e3df2[k3] + 1, nsealm)).astype(np.float32))
    fields.append(rng.standard_normal((p2[1] - p2[0] + 1, nsealm)).astype(np.float32))
    return {
        "ipar": ipar, "rpar": rpar, "flogrd": outg_flags(select, seed),
        "flogr2": outg_flags("some", seed + 1), "flogrr": outg_flags("some", seed + 2),
        "va": va, "nsealm": nsealm, "nsea": nsea,
        "cg": np.ascontiguousarray(cg, np.float32), "wn": np.ascontiguousarray(k, np.float32),
        "dw": dep.astype(np.float32), "sig": sig, "dden": dden, "dsii": dsii,
        "ecos": ecos, "esin": esin, "ec2": (ecos * ecos).astype(np.float32),
        "es2": (esin * esin).astype(np.float32), "esc": (ecos * esin).astype(np.float32),
        "mapsf": mapsf, "mapsta": mapsta, "fields": fields,
    }


def outg_part_case(nx=40, ny=30, seed=0, noswll=3, select="all", floutg2=0):
    """Seeded inputs of ww_outg_part: W3CPRT's ICPRT (NSEALM+1, 2) and DTPRT (15, NDTP) for the
    sea points of sea_grid (0 to 7 partitions a point, the first the whole spectrum; UNDEF in
    some directions; wind-sea fractions on both sides of WSCUT = 0.8), and 17 prefilled fields."""
    rng = np.random.default_rng(seed)
    mapsta, mapsf, nsea = sea_grid(nx, ny, seed=seed)
    nsealm = nsea + 1
    nicp = nsealm + 1
    n1 = rng.integers(0, 8, nicp).astype(np.int32)
    n2 = np.ones(nicp, np.int32)
    pos = 1
    for j in range(nicp):
        n2[j] = pos
        pos += max(int(n1[j]), 1)
    ndtp = pos - 1
    dtprt = rng.uniform(0.0, 20.0, (ndtp, 15)).astype(np.float32)
    dtprt[:, 5] = rng.uniform(0.0, 1.0, ndtp).astype(np.float32)
    undef = np.float32(-999.9)
    dtprt[rng.uniform(0, 1, ndtp) < 0.1, 3] = undef
    dtprt[rng.uniform(0, 1, ndtp) < 0.1, 6] = undef
    icprt = np.concatenate([n1, n2]).astype(np.int32)
    flog = np.zeros(OUTG_NOGRP * OUTG_NGRPP, np.int32)
    for j in range(1, 18):
        if select == "all" or rng.uniform() < 0.5:
            flog[3 + (j - 1) * OUTG_NOGRP] = 1
    ipar = np.array([nsea, nsea, nx, ny, nsealm, noswll, nicp, ndtp, 15, OUTG_NOGRP, OUTG_NGRPP,
                     1, floutg2], np.int32)
    fields = [rng.standard_normal((noswll + 1, nsealm)).astype(np.float32) for _ in range(15)]
    fields += [rng.standard_normal(nsealm).astype(np.float32) for _ in range(2)]
    return {"ipar": ipar, "rpar": np.array([undef, 0.8], np.float32), "flogrd": flog,
            "flogr2": outg_flags("none"), "mapsf": mapsf, "mapsta": mapsta, "icprt": icprt,
            "dtprt": np.ascontiguousarray(dtprt), "fields": fields, "nsea": nsea}
