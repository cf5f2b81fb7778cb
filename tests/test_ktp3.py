"""W3KTP3 (PR3/UQ spectral propagation with W3QCK1/W3QCK2) through the C ABI.

The checker is the reference's own C++ (kokkos/src/ww_kokkos/prop_ktp3.hpp with its shim
prop3_shim.cpp) compiled into oracle/_ref/libref_ww3.so and called through its C ABI
ww_ktp3_batch with the same arguments: the library's results must equal it bit for bit.
"""

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available
from oracle import oracle as _oracle

needs_ref = pytest.mark.skipif(not _oracle.ref_available(), reason="oracle/_ref not built")


@needs_ref
def test_reference_ktp3_runs_and_keeps_unlisted_columns(oracle, synth):
    c = synth.ktp3_case(200, seed=3, nsea=300)
    rc, va, cth, ck = oracle.ktp3_call(oracle.ref_lib(), c, itstep=1, ntimes=1)
    assert rc == 0
    listed = np.zeros(301, bool)
    listed[c["jsea"]] = True
    assert np.array_equal(va[~listed], c["va"][~listed])
    assert np.all(cth[c["jsea"] - 1] >= 0) and np.all(cth[~listed[1:]] == -1.0)


@needs_ref
def test_reference_ktp3_still_water_no_currents_keeps_directions(oracle, synth):
    """No depth gradient, no current, no great-circle turning: refraction velocity is zero, so
    only the wavenumber shift (also zero without currents) acts: the spectrum is unchanged."""
    c = synth.ktp3_case(50, seed=4, currents=False)
    ps = c["pscal"].reshape(-1, 10)
    ps[:, 0] = 0.0
    ps[:, 2:4] = 0.0
    c["pscal"] = ps.reshape(-1)
    rc, va, _, _ = oracle.ktp3_call(oracle.ref_lib(), c, itstep=2, ntimes=1)
    assert rc == 0
    assert_bitexact(va, c["va"], "still water")


@pytest.mark.parametrize("itstep,ntimes,currents", [(1, 1, True), (2, 1, True), (2, 2, False),
                                                    (3, 3, True)])
@needs_ref
@pytest.mark.gpu
def test_ktp3_gpu_bitexact(pkg, oracle, synth, itstep, ntimes, currents):
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    c = synth.ktp3_case(1500, seed=10 + itstep, nsea=2000, currents=currents)
    rc_r, va_r, cth_r, ck_r = oracle.ktp3_call(oracle.ref_lib(), c, itstep=itstep, ntimes=ntimes)
    rc, va, cth, ck = pkg.ktp3_batch(c, itstep=itstep, ntimes=ntimes)
    assert rc_r == 0 and rc == 0
    assert_bitexact(va, va_r, "VA")
    assert_bitexact(cth, cth_r, "CFLTHMAX")
    assert_bitexact(ck, ck_r, "CFLKMAX")



@needs_ref
@pytest.mark.gpu
def test_ktp3_resident_va_matches_host_form(pkg, oracle, synth):
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    c = synth.ktp3_case(800, seed=21, nsea=1000)
    va_host = np.array(c["va"], copy=True)
    rc_r, va_r, _, _ = oracle.ktp3_call(oracle.ref_lib(), c, itstep=2, ntimes=2)
    igrid = 77
    rc, _, _, _ = pkg.ktp3_batch(c, itstep=2, ntimes=2, igrid=igrid, va=va_host)
    assert rc == 0
    assert pkg.lib().ww_va_state(igrid) == 1  # DEVICE: the host copy is stale
    assert_bitexact(va_host, c["va"], "host VA untouched before the sync")
    assert pkg.va_host_read(igrid, va_host) == 0
    assert_bitexact(va_host, va_r, "VA after ww_va_host_read")
    assert pkg.lib().ww_va_state(igrid) == 2  # BOTH


@needs_ref
@pytest.mark.gpu
def test_ktp3_validation(pkg, synth):
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    c = synth.ktp3_case(10, seed=5)
    bad = dict(c)
    bad["rpar"] = c["rpar"][:2]
    assert pkg.ktp3_batch(bad)[0] == pkg.ERR_BAD_SHAPE
    bad = dict(c)
    bad["jsea"] = c["jsea"].copy()
    bad["jsea"][0] = 0
    rc, va, _, _ = pkg.ktp3_batch(bad)
    assert rc == pkg.ERR_BAD_SHAPE and np.array_equal(va, c["va"])
    bad = dict(c)
    bad["mapth2"] = c["mapth2"].copy()
    bad["mapth2"][5] = 10 ** 6
    assert pkg.ktp3_batch(bad)[0] == pkg.ERR_BAD_SHAPE
    zero = dict(c)
    zero["npts"] = 0
    rc, va, _, _ = pkg.ktp3_batch(zero)
    assert rc == pkg.OK and np.array_equal(va, c["va"])
