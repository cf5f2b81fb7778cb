"""W3MAP3 and W3MAPT on the device (ww_map3, ww_map3_device, ww_mapt) against the reference's
own builders (kokkos/src/ww_kokkos/prop_map3.hpp, prop_mapt.hpp, compiled into
oracle/_ref/libref_ww3.so): every list entry, every counter, the spectral maps and MAPTRN,
element for element, on seeded grids from 20 x 12 to the 1440 x 720 lon/lat grid of the
resident-step workload (0.72 M sea points), with boundary and excluded points."""

import numpy as np
import pytest

from conftest import cuda_available
from oracle import oracle as _oracle

needs_ref = pytest.mark.skipif(not _oracle.ref_available(), reason="oracle/_ref not built")

GRIDS = [(20, 12, 1), (48, 32, 2), (37, 29, 3), (1, 9, 4), (360, 180, 5), (1440, 720, 6)]
KEYS = ("mapx2", "mapy2", "mapaxy", "mapcxy", "mapth2", "mapwn2", "counts")


def _gpu():
    if not cuda_available():
        pytest.skip("needs a CUDA device")


def test_sea_grid_numbering(synth):
    sta, sf, nsea = synth.sea_grid(30, 20, seed=1)
    ix, iy, ixy = sf[:nsea], sf[nsea:2 * nsea], sf[2 * nsea:]
    assert np.array_equal(ixy, (ix - 1) * 20 + iy)
    assert np.all(sta[ixy - 1] != 0) and np.count_nonzero(sta) == nsea
    assert np.all(np.diff(iy * 1000 + ix) > 0)  # IY outer, IX inner
    assert {1, 2, -1} <= set(np.unique(sta[ixy - 1]).tolist())


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,seed", GRIDS)
def test_map3_equals_reference(pkg, synth, nx, ny, seed):
    _gpu()
    sta, sf, nsea = synth.sea_grid(nx, ny, seed=seed)
    nk, nth = 36, 36
    ref = _oracle.ref_w3map3_all(nx, ny, nsea, nk, nth, sta, sf)
    rc, got = pkg.map3(nx, ny, nsea, nk, nth, sta, sf)
    assert rc == 0
    for k in KEYS:
        assert np.array_equal(got[k], ref[k]), k


@needs_ref
@pytest.mark.gpu
def test_map3_keeps_set_spectral_maps_and_gtype3(pkg, synth):
    _gpu()
    sta, sf, nsea = synth.sea_grid(40, 24, seed=7)
    nk, nth = 12, 24
    preset = np.arange(1, (nk + 2) * nth + 1, dtype=np.int32)  # MAPTH2(1) /= 0: not rebuilt
    ref = _oracle.ref_w3map3_all(40, 24, nsea, nk, nth, sta, sf, mapth2=preset)
    rc, got = pkg.map3(40, 24, nsea, nk, nth, sta, sf, mapth2=preset)
    assert rc == 0
    for k in KEYS:
        assert np.array_equal(got[k], ref[k]), k
    assert np.array_equal(got["mapth2"], preset) and not got["mapwn2"].any()
    rc, got = pkg.map3(40, 24, nsea, nk, nth, sta, sf, gtype=3)  # no lists for GTYPE >= 3
    assert rc == 0 and not got["mapx2"].any() and not got["counts"].any()
    spectral = _oracle.ref_w3map3_all(40, 24, nsea, nk, nth, sta, sf)  # built from zeros
    assert np.array_equal(got["mapth2"], spectral["mapth2"])
    assert np.array_equal(got["mapwn2"], spectral["mapwn2"])


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,seed", [(48, 32, 2), (1440, 720, 6)])
def test_mapt_equals_reference(pkg, synth, nx, ny, seed):
    _gpu()
    sta, sf, nsea = synth.sea_grid(nx, ny, seed=seed)
    rng = np.random.default_rng(seed)
    nxy = nx * ny
    atrnx = rng.uniform(0.5, 1.0, 3 * nxy).astype(np.float32)
    atrny = rng.uniform(0.5, 1.0, 3 * nxy).astype(np.float32)
    atrnx[rng.uniform(0, 1, 3 * nxy) < 0.5] = 1.0
    atrnx[::997] = np.float32(float.fromhex('0x1.e66666p-1'))  # TRNMIN itself: not below it
    atrny[5::1009] = np.nan
    maptrn = (rng.uniform(0, 1, nxy) < 0.3).astype(np.int32)  # land cells keep theirs
    ref = _oracle.ref_w3mapt(nx, ny, nsea, sf, atrnx, atrny, maptrn)
    rc, got = pkg.mapt(nx, ny, nsea, sf, atrnx, atrny, maptrn)
    assert rc == 0 and np.array_equal(got, ref)


@pytest.mark.gpu
def test_map3_validation(pkg, synth):
    _gpu()
    sta, sf, nsea = synth.sea_grid(20, 12, seed=1)
    bad = sf.copy()
    bad[2 * nsea] += 1  # IXY no longer IY + (IX-1)*NY
    rc, got = pkg.map3(20, 12, nsea, 6, 8, sta, bad)
    assert rc == 2 and not got["counts"].any()
    bad = sf.copy()
    bad[0] = 21  # IX > NX
    rc, _ = pkg.map3(20, 12, nsea, 6, 8, sta, bad)
    assert rc == 2


def _utrn_inputs(synth, nx, ny, seed):
    sta, sf, nsea = synth.sea_grid(nx, ny, seed=seed)
    rng = np.random.default_rng(seed + 50)
    nxy = nx * ny
    trnx = np.where(rng.uniform(0, 1, nxy) < 0.8, 1.0, rng.uniform(0.0, 1.0, nxy)).astype(np.float32)
    trny = np.where(rng.uniform(0, 1, nxy) < 0.8, 1.0, rng.uniform(0.0, 1.0, nxy)).astype(np.float32)
    hpfac = rng.uniform(0.05, 0.5, nxy).astype(np.float32)
    hqfac = rng.uniform(0.05, 0.5, nxy).astype(np.float32)
    ice = np.where(rng.uniform(0, 1, nsea + 1) < 0.6, 0.0, rng.uniform(0.0, 1.0, nsea + 1))
    ice = ice.astype(np.float32)
    berg = np.where(rng.uniform(0, 1, nsea) < 0.9, 0.0, rng.uniform(0.0, 3.0, nsea))
    return sta, sf, nsea, trnx, trny, hpfac, hqfac, ice, berg.astype(np.float32)


# (trflag, fice0, ficen, ficel, ffacberg, flagll): every branch of W3UTRN
UTRN = [(0, 0.0, 0.0, 0.0, 0.0, 1), (1, 0.0, 0.0, 0.0, 0.0, 1), (2, 0.0, 0.0, 0.0, 0.0, 0),
        (3, 0.5, 0.75, 0.0, 10.0, 1), (4, 0.5, 0.75, 0.0, 10.0, 0), (5, 0.5, 0.75, 2.0e4, 5.0, 1),
        (3, 0.5, 0.5, 0.0, 10.0, 1)]


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("params", UTRN)
@pytest.mark.parametrize("nx,ny,seed", [(48, 32, 2), (1440, 720, 6)])
def test_utrn_equals_reference(pkg, synth, params, nx, ny, seed):
    _gpu()
    sta, sf, nsea, trnx, trny, hpfac, hqfac, ice, berg = _utrn_inputs(synth, nx, ny, seed)
    trflag, fice0, ficen, ficel, ffacberg, flagll = params
    args = (nx, ny, nsea, trflag, fice0, ficen, ficel, ffacberg, flagll, np.float32(0.625),
            trnx, trny, sf, sta, hpfac, hqfac, ice, berg)
    rx, ry = _oracle.ref_w3utrn(*args)
    rc, gx, gy = pkg.utrn(*args)
    assert rc == 0
    assert np.array_equal(gx.view(np.uint32), rx.view(np.uint32)), "ATRNX"
    assert np.array_equal(gy.view(np.uint32), ry.view(np.uint32)), "ATRNY"
