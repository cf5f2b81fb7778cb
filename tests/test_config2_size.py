"""The resident whole step at the sizes the workload names, bit for bit against the reference's
own C++ (oracle/_ref):

- W3XYP3 on the 1440 x 720 lon/lat grid (about 724,000 sea points, a VA of 9.4e8 floats) through
  the resident entry ww_xyp3_batch_va, on 16 spectral components spread over NSPEC (the `on`
  list, so the reference's CPU time stays bounded; every component runs the same code);
- W3KTP3 on every one of those sea points through ww_ktp3_batch_va;
- one recorded whole step (W3KTP3, W3XYP3, W3KTP3, W3SRCE with the bench's analytic-tail ST4
  and its own tables) replayed as a CUDA graph on a 360 x 180 grid (about 45,000 points).

At 1440 x 720 the spectra are U(0, 1) values, not sea states: what is under test there is the
index arithmetic of arrays near 2^30 elements, and both sides get the same values.
"""

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available
from oracle import oracle as _oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device"),
              pytest.mark.skipif(not _oracle.ref_available(), reason="oracle/_ref not built")]


@pytest.fixture(scope="module")
def grid1440(synth):
    return synth.xyp3_case(1440, 720, seed=61, ref=_oracle.ref_w3map3, spectra="uniform",
                           on_components=16)


def test_xyp3_1440x720_resident_bitexact(pkg, oracle, grid1440):
    c = grid1440
    assert c["nsea"] > 700_000
    rc_r, va_r = oracle.xyp3_call(oracle.ref_lib(), c)
    assert rc_r == 0
    va = np.array(c["va"], copy=True)
    rc, _ = pkg.xyp3_batch(c, igrid=91, va=va)
    assert rc == 0
    assert pkg.va_host_read(91, va) == 0
    assert_bitexact(va, va_r, "VA after W3XYP3 at 1440 x 720")
    on = np.nonzero(c["on"])[0]
    assert not np.array_equal(va[:, on], c["va"][:, on])  # the listed components moved


def test_ktp3_1440x720_resident_bitexact(pkg, oracle, synth, grid1440):
    nsea = grid1440["nsea"]
    c = synth.ktp3_case(nsea, seed=62, nsea=nsea, spectra="uniform")
    rc_r, va_r, cth_r, ck_r = oracle.ktp3_call(oracle.ref_lib(), c, itstep=1, ntimes=1)
    assert rc_r == 0
    va = np.array(c["va"], copy=True)
    rc, _, cth, ck = pkg.ktp3_batch(c, itstep=1, ntimes=1, igrid=92, va=va)
    assert rc == 0
    assert pkg.va_host_read(92, va) == 0
    assert_bitexact(va, va_r, "VA after W3KTP3 at 1440 x 720")
    assert_bitexact(cth, cth_r, "CFLTHMAX")
    assert_bitexact(ck, ck_r, "CFLKMAX")


def test_recorded_step_360x180_bitexact(pkg, oracle, synth):
    import test_step as ts

    st = synth.st4_setup(variant="analytic")
    t = synth.st4_tables_own(st)
    sr = synth.srce_setup(st)
    xc = synth.xyp3_case(360, 180, seed=71, ref=oracle.ref_w3map3)
    nsea = xc["nsea"]
    assert nsea > 40_000
    kc = synth.ktp3_case(nsea, seed=72, nsea=nsea)
    pts = synth.srce_points(nsea, seed=73)
    ref = oracle.RefSt4(st, t, igrid=751, srce=sr, dia=synth.dia_config(), scalar_mvec=True)
    c_ref = ts.Calls(ts._bind(ref.L), 751, np.array(xc["va"], np.float32, copy=True), kc, xc, pts)
    c_ref.step()
    va_ref = c_ref.read()
    L = ts._gpu_grid(pkg, oracle, synth, st, t, sr, 752)
    c_rec = ts.Calls(L, 752, np.array(xc["va"], np.float32, copy=True), kc, xc, pts)
    with pkg.Step(752) as step:
        c_rec.step()
    assert step.ops() == 4
    step.run(1)
    va_rec = c_rec.read()
    assert_bitexact(va_rec, va_ref, "VA after one recorded step at 360 x 180")
    step.free()
