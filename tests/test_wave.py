"""W3WAVE's per-step support routines through the reference's C ABI names (ww_wave_gath,
ww_wave_scat, ww_wave_uwnd, ww_wave_utrn, ww_wave_dzxy, ww_wave_map3, ww_wave_mapt,
ww_wave_distab, and ww_wave_cflxy for W3CFLXY, which the reference calls from its W3WAVE driver
only and is reached here through oracle/ref_driver.cpp's ref_w3cflxy) against the reference's
own shim (kokkos/src/fortran_iface/wave_support_shim.cpp
with its headers wave_gath_scat.hpp, updt_uwnd.hpp, updt_utrn.hpp, updt_dzxy.hpp, prop_map3.hpp,
prop_mapt.hpp, disp_distab.hpp, compiled into oracle/_ref/libref_ww3.so): every output element,
bit for bit, on seeded grids with MAPSF carrying more rows than sea points (MSEA > NSEA)."""

import ctypes

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available
from oracle import oracle as _oracle

P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
needs_ref = pytest.mark.skipif(not _oracle.ref_available(), reason="oracle/_ref not built")
OK, NOT_INIT, BAD_SHAPE = 0, 1, 2


def _bind(L):
    L.ww_wave_gath.argtypes = [I] * 7 + [P, P, P]
    L.ww_wave_scat.argtypes = [I] * 7 + [P, P, P, P]
    L.ww_wave_uwnd.argtypes = [I, F, F, I, F, I, I, I, I] + [P] * 20
    L.ww_wave_utrn.argtypes = [I, I, I, I, I, F, F, F, F, I] + [P] * 10
    L.ww_wave_dzxy.argtypes = [I, I, I] + [P] * 7 + [I, I, P, P]
    L.ww_wave_map3.argtypes = [I] * 7 + [P] * 9
    L.ww_wave_mapt.argtypes = [I, I, I, P, P, P, P]
    L.ww_wave_distab.argtypes = [I, P, P, P, P]
    for n in ("gath", "scat", "uwnd", "utrn", "dzxy", "map3", "mapt", "distab"):
        getattr(L, "ww_wave_" + n).restype = I
    return L


def _ref():
    return _bind(_oracle.ref_lib())


def _gpu(pkg):
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    L = pkg.lib()
    pkg.init()
    return _bind(L)


def p(x):
    return x.ctypes.data


def grid(synth, nx, ny, seed, extra=3):
    """MAPSTA (NY,NX), MAPSF padded to MSEA = NSEA + extra rows (the padding is junk), NSEA."""
    sta, sf, nsea = synth.sea_grid(nx, ny, seed=seed)
    msea = nsea + extra
    m = np.full((3, msea), -7, np.int32)
    m[:, :nsea] = sf.reshape(3, nsea)
    return sta, np.ascontiguousarray(m.reshape(-1)), nsea, msea


def both(pkg, fn):
    """fn(L) on the reference and on the library; returns (reference result, device result)."""
    L = _gpu(pkg)
    return fn(_ref()), fn(L)


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,seed", [(24, 18, 1), (61, 40, 2)])
def test_gath_scat(pkg, synth, nx, ny, seed):
    sta, sf, nsea, msea = grid(synth, nx, ny, seed)
    rng = np.random.default_rng(seed)
    nspec, ncol = 24, nsea + 3
    va0 = rng.standard_normal((ncol, nspec)).astype(np.float32)
    nf = ny * (nx + 3)
    for ispec in (1, 7, nspec):
        def gath(L):
            f = np.full(nf, 123.0, np.float32)
            assert L.ww_wave_gath(ispec, nspec, nsea, ncol, msea, nx, ny, p(va0), p(sf), p(f)) == OK
            return f
        r, d = both(pkg, gath)
        assert_bitexact(d, r, f"W3GATH ispec {ispec}")
        field = rng.standard_normal(nf).astype(np.float32)

        def scat(L):
            va = va0.copy()
            assert L.ww_wave_scat(ispec, nspec, nsea, ncol, msea, nx, ny, p(sta), p(field), p(sf),
                                  p(va)) == OK
            return va
        r, d = both(pkg, scat)
        assert_bitexact(d, r, f"W3SCAT ispec {ispec}")
        assert not np.array_equal(r, va0)


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("flfrst,flcur", [(1, 0), (1, 1), (0, 0), (0, 1)])
def test_uwnd(pkg, synth, flfrst, flcur):
    nx, ny = 37, 23
    sta, sf, nsea, msea = grid(synth, nx, ny, 5)
    rng = np.random.default_rng(11 + flfrst + 2 * flcur)
    fld = {k: rng.uniform(-25, 25, (ny, nx)).astype(np.float32) for k in ("wx0", "wy0", "wxn", "wyn")}
    calm = rng.uniform(0, 1, (ny, nx)) < 0.05
    fld["wx0"][calm] = 0.0
    fld["wy0"][calm] = 0.0
    fld["wxn"][rng.uniform(0, 1, (ny, nx)) < 0.05] = 0.0
    fld["dt0"] = rng.uniform(-3, 3, (ny, nx)).astype(np.float32)
    fld["dtn"] = rng.uniform(-3, 3, (ny, nx)).astype(np.float32)
    # WX0(NX,NY): the (NY,NX) C arrays hold the Fortran order
    fld = {k: np.ascontiguousarray(v) for k, v in fld.items()}
    cx = rng.uniform(-1, 1, nsea).astype(np.float32)
    cy = rng.uniform(-1, 1, nsea).astype(np.float32)
    state0 = [rng.uniform(0, 6, nsea).astype(np.float32) for _ in range(11)]

    def call(L):
        st = [s.copy() for s in state0]
        rc = L.ww_wave_uwnd(flfrst, 3600.0, 1200.0, flcur, 0.7, nsea, msea, nx, ny, p(sf),
                            *[p(fld[k]) for k in ("wx0", "wy0", "dt0", "wxn", "wyn", "dtn")],
                            p(cx), p(cy), *[p(s) for s in st])
        assert rc == OK
        return st
    r, d = both(pkg, call)
    names = "UA0 UAI UD0 UDI AS0 ASI UA UD AS U10 U10D".split()
    for k in range(11):
        assert_bitexact(d[k], r[k], f"W3UWND {names[k]}")


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("trflag", [0, 1, 2, 3, 4, 5])
def test_utrn(pkg, synth, trflag):
    nx, ny = 30, 20
    sta, sf, nsea, msea = grid(synth, nx, ny, 7)
    rng = np.random.default_rng(20 + trflag)
    nc = nx * ny
    trnx = rng.uniform(0, 1, nc).astype(np.float32)
    trny_ext = rng.uniform(0, 1, nc + 1).astype(np.float32)  # element 0 is the REAL before TRNY
    hp = rng.uniform(1e3, 3e4, nc).astype(np.float32)
    hq = rng.uniform(1e3, 3e4, nc).astype(np.float32)
    ice = rng.uniform(0, 1, nsea + 1).astype(np.float32)
    ice[rng.uniform(0, 1, nsea + 1) < 0.5] = 0.0
    berg = rng.uniform(0, 2, nsea).astype(np.float32)
    berg[rng.uniform(0, 1, nsea) < 0.7] = 0.0

    def call(L):
        ax = np.zeros(3 * nc, np.float32)
        ay = np.zeros(3 * nc, np.float32)
        rc = L.ww_wave_utrn(nx, ny, nsea, msea, trflag, 0.25, 0.75, 0.0 if trflag < 4 else 1.5,
                            0.3, 1, p(trnx), trny_ext.ctypes.data + 4, p(sf), p(sta), p(hp),
                            p(hq), p(ice), p(berg), p(ax), p(ay))
        assert rc == OK
        return ax, ay
    r, d = both(pkg, call)
    assert_bitexact(d[0], r[0], f"ATRNX trflag {trflag}")
    assert_bitexact(d[1], r[1], f"ATRNY trflag {trflag}")


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("iclose,flagll", [(-1, 1), (2, 1), (8, 0), (2, 0)])
def test_dzxy(pkg, synth, iclose, flagll):
    nx, ny = 44, 31
    sta, sf, nsea, msea = grid(synth, nx, ny, 9)
    rng = np.random.default_rng(30 + iclose)
    mapfs = np.zeros(nx * ny, np.int32)
    mapfs[sf[2 * msea:2 * msea + nsea] - 1] = np.arange(1, nsea + 1, dtype=np.int32)
    zz = rng.uniform(5, 4000, nsea).astype(np.float32)
    met = [rng.uniform(-2, 2, nx * ny).astype(np.float32) for _ in range(4)]

    def call(L):
        gx = np.full(nx * ny, 9.0, np.float32)
        gy = np.full(nx * ny, 9.0, np.float32)
        rc = L.ww_wave_dzxy(nsea, nx, ny, p(zz), p(sta), p(mapfs), *[p(m) for m in met], flagll,
                            iclose, p(gx), p(gy))
        assert rc == OK
        return gx, gy
    r, d = both(pkg, call)
    assert_bitexact(d[0], r[0], "DZZDX")
    assert_bitexact(d[1], r[1], "DZZDY")


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,seed,gtype", [(20, 12, 1, 1), (48, 32, 2, 2), (37, 29, 3, 1)])
def test_map3_mapt(pkg, synth, nx, ny, seed, gtype):
    sta, sf, nsea, msea = grid(synth, nx, ny, seed)
    nk, nth = 12, 8
    nc = nx * ny
    rng = np.random.default_rng(seed)

    def call(L):
        m = {k: np.full(n, -5, np.int32) for k, n in (("x2", nc), ("y2", nc), ("axy", nc),
                                                       ("cxy", nsea), ("th2", (nk + 2) * nth),
                                                       ("wn2", nk * nth + nth))}
        counts = np.zeros(8, np.int32)
        rc = L.ww_wave_map3(nx, ny, nsea, msea, nk, nth, gtype, p(sta), p(sf), p(m["x2"]),
                            p(m["y2"]), p(m["axy"]), p(m["cxy"]), p(m["th2"]), p(m["wn2"]),
                            p(counts))
        assert rc == OK
        return m, counts
    r, d = both(pkg, call)
    for k in r[0]:
        assert_bitexact(d[0][k], r[0][k], f"W3MAP3 {k}")
    assert_bitexact(d[1], r[1], "W3MAP3 counts")
    ax = rng.uniform(0, 1, 3 * nc).astype(np.float32)
    ay = rng.uniform(0, 1, 3 * nc).astype(np.float32)
    ax[rng.uniform(0, 1, 3 * nc) < 0.3] = 1.0

    def mapt(L):
        t = rng.integers(0, 2, nc).astype(np.int32) * 0 + 3
        assert L.ww_wave_mapt(nsea, msea, nc, p(sf), p(ax), p(ay), p(t)) == OK
        return t
    r, d = both(pkg, mapt)
    assert_bitexact(d, r, "W3MAPT")


@needs_ref
@pytest.mark.gpu
def test_distab(pkg):
    def call(L):
        w = np.zeros(122, np.float32)
        c = np.zeros(122, np.float32)
        n1 = np.zeros(1, np.int32)
        ds = np.zeros(1, np.float32)
        assert L.ww_wave_distab(121, p(w), p(c), p(n1), p(ds)) == OK
        return w, c, n1, ds
    r, d = both(pkg, call)
    for k, name in enumerate(("EWN1", "ECG1", "N1MAX", "DSIE")):
        assert_bitexact(d[k], r[k], f"DISTAB {name}")
    assert int(d[2][0]) == 120 and np.all(np.diff(d[0][1:]) > 0)


# ------------------------------------------------------------ host checks (no device needed)
@needs_ref
def test_wave_statuses_match_reference(pkg, synth):
    L = _bind(pkg.lib())
    R = _ref()
    sta, sf, nsea, msea = grid(synth, 20, 12, 1)
    va = np.zeros((nsea + 1, 4), np.float32)
    f = np.zeros(12 * 23, np.float32)
    for X in (L, R):
        assert X.ww_wave_gath(0, 4, nsea, nsea + 1, msea, 20, 12, p(va), p(sf), p(f)) == BAD_SHAPE
        assert X.ww_wave_scat(1, 4, nsea, nsea, msea, 20, 12, p(sta), p(f), p(sf), p(va)) == BAD_SHAPE
        assert X.ww_wave_map3(20, 12, nsea, msea, 6, 4, 3, p(sta), p(sf), *[p(f)] * 7) == BAD_SHAPE
        assert X.ww_wave_distab(120, p(f), p(f), p(f), p(f)) == BAD_SHAPE
        assert X.ww_wave_mapt(nsea, nsea - 1, 240, p(sf), p(f), p(f), p(f)) == BAD_SHAPE
    if not cuda_available():
        assert L.ww_wave_gath(1, 4, nsea, nsea + 1, msea, 20, 12, p(va), p(sf), p(f)) == NOT_INIT
    bad = sf.copy()
    bad[2 * msea] = 20 * 12 + 1  # the library refuses a cell outside the grid
    assert L.ww_wave_gath(1, 4, nsea, nsea + 1, msea, 20, 12, p(va), p(bad), p(f)) == BAD_SHAPE


def _cflxy_case(synth, nx, ny, nk, nth, seed, ties):
    """A seeded W3CFLXY case on a synthetic grid; ties=True plants zero group velocities and
    signed-zero metric terms so that the MAX operand order decides the sign of zero results."""
    sta, sf, nsea, msea = grid(synth, nx, ny, seed)
    rng = np.random.default_rng(seed + 40)
    th = (np.arange(nth) + 0.5) * (2 * np.pi / nth)
    ecos = np.cos(th).astype(np.float32)
    esin = np.sin(th).astype(np.float32)
    clats = rng.uniform(0.2, 1.0, nsea + 1).astype(np.float32)
    met = [rng.uniform(-4e-4, 4e-4, nx * ny).astype(np.float32) for _ in range(4)]
    cg = rng.uniform(0.5, 25.0, (nsea + 1, nk + 2)).astype(np.float32)
    cx = rng.uniform(-1.5, 1.5, nsea + 1).astype(np.float32)
    cy = rng.uniform(-1.5, 1.5, nsea + 1).astype(np.float32)
    if ties:
        cg[1::5, :] = 0.0  # every fifth point: no advection, all CFL numbers are +-0
        for m in met:
            m[::7] = -0.0
        cx[::3] = 0.0
        cy[::3] = -0.0
    return sf, nsea, msea, clats, ecos, esin, met, np.ascontiguousarray(cg.reshape(-1)), cx, cy


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("nk,nth,flcur,mgp,ties", [
    (36, 36, 0, 0, False), (36, 36, 1, 0, False), (36, 36, 0, 0, True), (36, 36, 1, 0, True),
    (5, 7, 0, 0, True), (5, 7, 1, 0, True), (5, 7, 1, 1, True), (4, 1, 0, 0, True),
    (4, 1, 0, 1, True), (4, 1, 1, 0, True), (3, 2, 0, 1, True)])
def test_cflxy(pkg, synth, nk, nth, flcur, mgp, ties):
    nx, ny = 41, 29
    sf, nsea, msea, clats, ecos, esin, met, cg, cx, cy = _cflxy_case(synth, nx, ny, nk, nth,
                                                                      nk * 10 + nth, ties)
    dtg, vgx, vgy = 900.0, 0.75, -0.5
    L = _gpu(pkg)
    L.ww_wave_cflxy.argtypes = [I] * 9 + [F, F, F] + [P] * 12
    L.ww_wave_cflxy.restype = I
    R = _oracle.ref_lib()
    R.ref_w3cflxy.argtypes = [I] * 7 + [F, F, F] + [P] * 12
    R.ref_w3cflxy.restype = I
    sf_n = np.ascontiguousarray(sf.reshape(3, msea)[:, :nsea].reshape(-1))
    ref = np.full(nsea, 7.0, np.float32)
    assert R.ref_w3cflxy(nsea, nx, ny, nk, nth, flcur, mgp, dtg, vgx, vgy, p(sf_n), p(clats),
                         p(ecos), p(esin), *[p(m) for m in met], p(cg), p(cx), p(cy),
                         p(ref)) == 0
    dev = np.full(nsea, 7.0, np.float32)
    rc = L.ww_wave_cflxy(0, nsea, msea, nx, ny, nk, nth, flcur, mgp, dtg, vgx, vgy, p(sf),
                         p(clats), p(ecos), p(esin), *[p(m) for m in met], p(cg), p(cx), p(cy),
                         p(dev))
    assert rc == OK
    assert_bitexact(dev, ref, f"CFLXYMAX nk {nk} nth {nth} flcur {flcur} mgp {mgp}")
    assert np.all(ref >= 0)  # CFLXYMAX starts at 0
    if ties and not mgp:
        assert np.any(ref == 0)


def test_cflxy_refuses_bad_maps(pkg, synth):
    """A MAPSF entry off the grid is BAD_SHAPE before any device work (no GPU needed)."""
    L = pkg.lib()
    L.ww_wave_cflxy.argtypes = [I] * 9 + [F, F, F] + [P] * 12
    L.ww_wave_cflxy.restype = I
    nx, ny, nk, nth = 12, 9, 3, 4
    sf, nsea, msea, clats, ecos, esin, met, cg, cx, cy = _cflxy_case(synth, nx, ny, nk, nth, 5,
                                                                      False)
    sf = sf.copy()
    sf[msea + 1] = ny + 1
    out = np.zeros(nsea, np.float32)
    rc = L.ww_wave_cflxy(0, nsea, msea, nx, ny, nk, nth, 0, 0, 900.0, 0.0, 0.0, p(sf), p(clats),
                         p(ecos), p(esin), *[p(m) for m in met], p(cg), None, None, p(out))
    assert rc == BAD_SHAPE


@needs_ref
@pytest.mark.gpu
def test_cflxy_on_a_propagation_case(pkg, synth):
    """W3CFLXY on the arrays of a W3XYP3 case (regular 0.25-degree grid, currents on, NK = NTH =
    36): the module arrays exactly as the propagation reads them."""
    xc = synth.xyp3_case(48, 32, seed=7, ref=_oracle.ref_w3map3)
    ip = xc["ipar"]
    nx, ny, nsea, nk, nth, flcur = (int(ip[i]) for i in (0, 1, 2, 3, 4, 10))
    arrs = [np.ascontiguousarray(xc[a]) for a in ("mapsf", "clats", "ecos", "esin", "dpdx",
                                                  "dpdy", "dqdx", "dqdy", "cg", "cx", "cy")]
    L = _gpu(pkg)
    L.ww_wave_cflxy.argtypes = [I] * 9 + [F, F, F] + [P] * 12
    L.ww_wave_cflxy.restype = I
    R = _oracle.ref_lib()
    R.ref_w3cflxy.argtypes = [I] * 7 + [F, F, F] + [P] * 12
    R.ref_w3cflxy.restype = I
    ref = np.zeros(nsea, np.float32)
    assert R.ref_w3cflxy(nsea, nx, ny, nk, nth, flcur, 0, xc["dtg"], 0.0, 0.0,
                         *[p(a) for a in arrs], p(ref)) == 0
    dev = np.zeros(nsea, np.float32)
    assert L.ww_wave_cflxy(0, nsea, nsea, nx, ny, nk, nth, flcur, 0, xc["dtg"], 0.0, 0.0,
                           *[p(a) for a in arrs], p(dev)) == OK
    assert_bitexact(dev, ref, "CFLXYMAX, propagation case")
    assert ref.max() > 0


@needs_ref
@pytest.mark.parametrize("flcur,mgp", [(0, 0), (1, 0), (1, 1)])
def test_ref_cflxy_is_the_formula(synth, flcur, mgp):
    """The reference's W3CFLXY as oracle/ref_driver.cpp binds it equals the routine's formula
    (w3pro3md.F90:2105-2128) restated in float32 numpy, up to the sign of zero: pins the driver's
    array layouts (MAPSF, CG, the metric fields) before the device is compared with it."""
    nx, ny, nk, nth = 23, 17, 6, 9
    sf, nsea, msea, clats, ecos, esin, met, cg, cx, cy = _cflxy_case(synth, nx, ny, nk, nth, 3,
                                                                      False)
    dtg, vgx, vgy = np.float32(600.0), np.float32(0.3), np.float32(-0.2)
    R = _oracle.ref_lib()
    R.ref_w3cflxy.argtypes = [I] * 7 + [F, F, F] + [P] * 12
    R.ref_w3cflxy.restype = I
    sf_n = np.ascontiguousarray(sf.reshape(3, msea)[:, :nsea].reshape(-1))
    ref = np.zeros(nsea, np.float32)
    assert R.ref_w3cflxy(nsea, nx, ny, nk, nth, flcur, mgp, float(dtg), float(vgx), float(vgy),
                         p(sf_n), p(clats), p(ecos), p(esin), *[p(m) for m in met], p(cg), p(cx),
                         p(cy), p(ref)) == 0
    isea = np.arange(1, nsea + 1)
    ixy = (sf_n[:nsea] - 1) * ny + (sf_n[nsea:2 * nsea] - 1)
    dpdx, dpdy, dqdx, dqdy = (m[ixy][:, None, None] for m in met)
    cl = clats[isea][:, None, None]
    cgk = cg.reshape(nsea + 1, nk + 2)[isea, 1:nk + 1][:, :, None]
    cxt = (ecos[None, None, :] * cgk) / cl
    cyt = esin[None, None, :] * cgk
    if mgp:
        cxt, cyt = cxt - vgx / cl, cyt - vgy
    if flcur:
        cxt = cxt + cx[isea][:, None, None] / cl
        cyt = cyt + cy[isea][:, None, None]
    vx = (cxt * dpdx + cyt * dpdy) * dtg
    vy = (cxt * dqdx + cyt * dqdy) * dtg
    want = np.maximum(np.maximum(vx, vy).max(axis=(1, 2)), np.float32(0))
    assert want.dtype == np.float32
    np.testing.assert_array_equal(ref, want)
