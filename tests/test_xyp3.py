"""W3XYP3 (PR3/UQ spatial propagation with W3QCK3, W3GATH and W3SCAT) through the C ABI.

The checker is the reference's own C++ (kokkos/src/ww_kokkos/prop_xyp3.hpp with its shim
prop3_shim.cpp, the averaging run serially in source order) compiled into
oracle/_ref/libref_ww3.so and called through its C ABI ww_xyp3_batch with the same arguments.
The library's averaging is an ordered gather per target cell; its results must equal the
reference's bit for bit. The grids are seeded land/sea masks with active boundary points,
excluded sea points, transparencies, averaging switched off on some cells (MAPTRN), currents
and boundary input (one point listed twice), built with the reference's own W3MAP3.
"""

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available
from oracle import oracle as _oracle

needs_ref = pytest.mark.skipif(not _oracle.ref_available(), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def maps():
    return _oracle.ref_w3map3


@needs_ref
def test_reference_w3map3_maps_are_consistent(synth, maps):
    c = synth.xyp3_case(40, 24, seed=2, ref=maps)
    counts = c["imaps"]
    nsea = c["nsea"]
    assert sorted(c["mapcxy"].tolist()) == list(range(1, nsea + 1))
    assert 0 < counts[7] < nsea  # central and near-coast points both present
    assert counts[0] <= counts[1] <= counts[2] and counts[3] <= counts[4] <= counts[5]


@needs_ref
def test_reference_xyp3_runs(oracle, synth, maps):
    c = synth.xyp3_case(40, 24, seed=3, ref=maps)
    rc, va = oracle.xyp3_call(oracle.ref_lib(), c)
    assert rc == 0 and np.isfinite(va).all()
    assert np.any(va != c["va"])


CASES = [
    dict(nx=48, ny=32, seed=1, iclose=2, flcur=True, flbpi=True),
    dict(nx=203, ny=77, seed=5, iclose=2, flcur=True, flbpi=False, on_fraction=0.1),
    dict(nx=48, ny=32, seed=2, iclose=-1, flcur=False, flbpi=False),
    dict(nx=37, ny=29, seed=3, iclose=2, flcur=True, flbpi=True, on_fraction=0.5),
    dict(nx=60, ny=20, seed=4, iclose=-1, flcur=True, flbpi=True, dtg=3600.0),
]


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_xyp3_gpu_bitexact(pkg, oracle, synth, maps, case):
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    c = synth.xyp3_case(ref=maps, **case)
    rc_r, va_r = oracle.xyp3_call(oracle.ref_lib(), c)
    rc, va = pkg.xyp3_batch(c)
    assert rc_r == 0 and rc == 0
    assert_bitexact(va, va_r, "VA after W3XYP3")


@needs_ref
@pytest.mark.gpu
def test_xyp3_resident_then_ktp3(pkg, oracle, synth, maps):
    """The resident VA across a propagation step: XYP3 then a host read equals the reference."""
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    c = synth.xyp3_case(48, 32, seed=7, ref=maps)
    rc_r, va_r = oracle.xyp3_call(oracle.ref_lib(), c)
    va = np.array(c["va"], copy=True)
    igrid = 88
    rc, _ = pkg.xyp3_batch(c, igrid=igrid, va=va)
    assert rc == 0 and pkg.lib().ww_va_state(igrid) == 1
    assert pkg.va_host_read(igrid, va) == 0
    assert_bitexact(va, va_r, "resident VA after W3XYP3")


@needs_ref
@pytest.mark.gpu
def test_xyp3_validation(pkg, synth, maps):
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    c = synth.xyp3_case(40, 24, seed=5, ref=maps)
    bad = dict(c)
    bad["ipar"] = c["ipar"].copy()
    bad["ipar"][6] = 8  # tripole
    assert pkg.xyp3_batch(bad)[0] == pkg.ERR_UNSUPPORTED
    bad = dict(c)
    bad["mapcxy"] = c["mapcxy"].copy()
    bad["mapcxy"][0] = bad["mapcxy"][1]
    rc, va = pkg.xyp3_batch(bad)
    assert rc == pkg.ERR_BAD_SHAPE and np.array_equal(va, c["va"])
    bad = dict(c)
    bad["rpar"] = c["rpar"][:4]
    assert pkg.xyp3_batch(bad)[0] == pkg.ERR_BAD_SHAPE


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("case", [CASES[0], CASES[2], CASES[4]])
def test_xyp3_list_sweeps_bitexact(pkg, oracle, synth, maps, case, monkeypatch):
    """The sweeps as list kernels (WW_B200_XYP3_LISTS=1, one thread per MAPX2/MAPY2/MAPAXY
    entry) and tiled in shared memory (the default) both give the reference's bits."""
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    c = synth.xyp3_case(ref=maps, **case)
    rc_r, va_r = oracle.xyp3_call(oracle.ref_lib(), c)
    monkeypatch.setenv("WW_B200_XYP3_LISTS", "1")
    rc, va_l = pkg.xyp3_batch(c)
    monkeypatch.delenv("WW_B200_XYP3_LISTS")
    rc2, va_t = pkg.xyp3_batch(c)
    assert rc_r == 0 and rc == 0 and rc2 == 0
    assert_bitexact(va_l, va_r, "VA after W3XYP3, list sweeps")
    assert_bitexact(va_t, va_r, "VA after W3XYP3, tiled sweeps")
