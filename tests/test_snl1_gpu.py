"""W3SNL1 on the GPU through the C ABI, bit for bit against the CPU oracle.

The bar is bit-exactness (float32, same operation order, no fused multiply-add): every S and D
value of the CUDA kernels equals the oracle's, which the CPU tests pin to the Fortran golden
vector and to the reference's own C++ build.
"""

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

KERNELS = ["gather", "rowshift", "band", "tile", "pair", "pair-general"]


def kernel_id(pkg, name):
    return {"gather": pkg.KERNEL_GATHER, "rowshift": pkg.KERNEL_ROWSHIFT,
            "band": pkg.KERNEL_BAND, "tile": pkg.KERNEL_TILE, "pair": pkg.KERNEL_PAIR,
            "pair-general": pkg.KERNEL_PAIR_GENERAL}[name]


def try_select(pkg, grid, name):
    """Select kernel `name`; False when its instances do not fit the grid (only the tile
    kernel, whose instances need 36 or 24 directions and NK a multiple of 4, and the pair
    kernel, whose bulk copies need NSPEC and NK multiples of 4)."""
    try:
        grid.select_kernel(kernel_id(pkg, name))
    except ValueError:
        assert name in ("tile", "pair", "pair-general")
        return False
    return True


@pytest.fixture(scope="module")
def cfg36(synth):
    return synth.dia_config()


def test_golden_vector_with_fortran_tables(pkg, golden):
    """The Fortran's own INSNL1 tables imported through ww_snl1_init_tables: the GPU reproduces
    the Fortran W3SNL1 answers of the golden vector bit for bit, on both kernels."""
    tables = {k: golden[k] for k in ("scal", "wts", "ipim", "ic", "af11")}
    grid = pkg.Snl1Grid(golden["cfg"], golden["sig"], igrid=31, tables=tables)
    for name in KERNELS:
        if not try_select(pkg, grid, name):
            continue
        s, d = grid(golden["a"], golden["cg"], golden["kdmean"])
        assert_bitexact(s, golden["s"], f"S vs Fortran ({name})")
        assert_bitexact(d, golden["d"], f"D vs Fortran ({name})")


def test_golden_inputs_with_built_tables(pkg, oracle, golden):
    grid = pkg.Snl1Grid(golden["cfg"], golden["sig"], igrid=32)
    s_ref, d_ref = oracle.w3snl1(golden["cfg"], golden["sig"], golden["a"], golden["cg"],
                                 golden["kdmean"])
    for name in KERNELS:
        if not try_select(pkg, grid, name):
            continue
        s, d = grid(golden["a"], golden["cg"], golden["kdmean"])
        assert_bitexact(s, s_ref, f"S ({name})")
        assert_bitexact(d, d_ref, f"D ({name})")


@pytest.mark.parametrize("name", KERNELS)
@pytest.mark.parametrize("case", ["deep", "mixed", "shallow", "bimodal"])
def test_36x36_bitexact(pkg, oracle, synth, cfg36, name, case):
    kw = {"deep": {}, "mixed": {"depth_range": (5.0, 4000.0)},
          "shallow": {"depth_range": (0.5, 15.0)},
          "bimodal": {"depth_range": (5.0, 4000.0), "bimodal": 0.5}}[case]
    cfg, sig = cfg36
    g = synth.sea_states(1000, seed=1234, **kw)
    grid = pkg.Snl1Grid(cfg, sig, igrid=1)
    grid.select_kernel(kernel_id(pkg, name))
    s, d = grid(g["a"], g["cg"], g["kdmean"])
    s_ref, d_ref = oracle.w3snl1(cfg, sig, g["a"], g["cg"], g["kdmean"])
    assert_bitexact(s, s_ref, "S")
    assert_bitexact(d, d_ref, "D")


@pytest.mark.parametrize("name", ["band", "pair", "pair-general"])
@pytest.mark.parametrize("npts", [1, 2, 3, 287, 8191, 8192, 8193, 20000])
def test_ragged_batch_sizes(pkg, oracle, synth, cfg36, npts, name):
    """Sizes around the host pipeline's chunk (8192 points), the CTA count and, for the pair
    kernel, odd counts (the last point paired with itself and stored once)."""
    cfg, sig = cfg36
    g = synth.sea_states(npts, seed=npts, depth_range=(5.0, 4000.0))
    grid = pkg.Snl1Grid(cfg, sig, igrid=2)
    grid.select_kernel(kernel_id(pkg, name))
    s, d = grid(g["a"], g["cg"], g["kdmean"])
    s_ref, d_ref = oracle.w3snl1(cfg, sig, g["a"], g["cg"], g["kdmean"])
    assert_bitexact(s, s_ref, "S")
    assert_bitexact(d, d_ref, "D")


@pytest.mark.parametrize("nk,nth", [(25, 24), (28, 24), (30, 36), (36, 36), (32, 48), (40, 72), (36, 13)])
def test_other_spectral_grids(pkg, oracle, nk, nth):
    rng = np.random.default_rng(nk * 100 + nth)
    sig = (2 * np.pi * 0.04 * 1.1 ** np.arange(nk)).astype(np.float32)
    cfg = {"nk": nk, "nth": nth, "xfr": float(np.float32(1.1)),
           "dth": float(np.float32(2 * np.pi / nth)), "lam": 0.25,
           "snlc1": float(np.float32(2.78e7 / 9.806 ** 4)), "kdcon": 0.75, "kdmn": 0.5,
           "snls1": 5.5, "snls2": float(np.float32(0.833)), "snls3": -1.25,
           "fachfe": float(np.float32(1.1) ** np.float32(-5))}
    npts = 300
    a = (rng.random((npts, nk * nth)) * 1e-3).astype(np.float32)
    cg = (rng.random((npts, nk)) * 10 + 1).astype(np.float32)
    kd = (rng.random(npts) * 20 + 0.1).astype(np.float32)
    grid = pkg.Snl1Grid(cfg, sig, igrid=100 + nth)
    s_ref, d_ref = oracle.w3snl1(cfg, sig, a, cg, kd)
    for name in KERNELS:
        try:
            grid.select_kernel(kernel_id(pkg, name))
        except ValueError:
            assert name in ("rowshift", "band", "tile", "pair", "pair-general")
            continue
        s, d = grid(a, cg, kd)
        assert_bitexact(s, s_ref, f"S {nk}x{nth} {name}")
        assert_bitexact(d, d_ref, f"D {nk}x{nth} {name}")


def test_device_entry_matches_host_entry(pkg, synth, cfg36):
    import torch

    cfg, sig = cfg36
    g = synth.sea_states(5000, seed=5, depth_range=(5.0, 4000.0))
    grid = pkg.Snl1Grid(cfg, sig, igrid=3)
    s_h, d_h = grid(g["a"], g["cg"], g["kdmean"])
    dev = torch.device("cuda:0")
    a = torch.from_numpy(g["a"]).to(dev)
    cg = torch.from_numpy(g["cg"]).to(dev)
    kd = torch.from_numpy(g["kdmean"]).to(dev)
    s = torch.full_like(a, float("nan"))
    d = torch.full_like(a, float("nan"))
    stream = torch.cuda.current_stream().cuda_stream
    grid.run_device(a.shape[0], a, cg, kd, s, d, stream)
    torch.cuda.synchronize()
    assert_bitexact(s.cpu().numpy(), s_h, "S device vs host entry")
    assert_bitexact(d.cpu().numpy(), d_h, "D device vs host entry")


def test_npts_zero_and_validation(pkg, synth, cfg36):
    cfg, sig = cfg36
    grid = pkg.Snl1Grid(cfg, sig, igrid=4)
    L = pkg.lib()
    a = np.zeros((3, 1296), np.float32)
    s = np.full_like(a, 5.0)
    L.ww_snl1(4, 0, a.ctypes.data, a.ctypes.data, a.ctypes.data, s.ctypes.data, s.ctypes.data)
    assert pkg.last_error() == pkg.OK and np.all(s == 5.0)
    L.ww_snl1(4, -1, a.ctypes.data, a.ctypes.data, a.ctypes.data, s.ctypes.data, s.ctypes.data)
    assert pkg.last_error() == pkg.ERR_BAD_SHAPE and np.all(s == 5.0)
    L.ww_snl1(4, 3, a.ctypes.data, None, a.ctypes.data, s.ctypes.data, s.ctypes.data)
    assert pkg.last_error() == pkg.ERR_BAD_SHAPE and np.all(s == 5.0)
    assert L.ww_snl1_init(5, 0, 36, *([1.0] * 10), sig) == pkg.ERR_BAD_SHAPE
    L.ww_snl1(5, 3, a.ctypes.data, a.ctypes.data, a.ctypes.data, s.ctypes.data, s.ctypes.data)
    assert pkg.last_error() == pkg.ERR_NOT_INITIALISED  # a failed init leaves no grid
    grid(np.ones((2, 1296), np.float32), np.ones((2, 36), np.float32),
         np.ones(2, np.float32))
    assert pkg.last_error() == pkg.OK


def test_bad_imported_tables_are_refused(pkg, golden):
    tables = {k: golden[k].copy() for k in ("scal", "wts", "ipim", "ic", "af11")}
    tables["ipim"][3, 10] = 10 ** 6
    with pytest.raises(pkg.WwError) as e:
        pkg.Snl1Grid(golden["cfg"], golden["sig"], igrid=33, tables=tables)
    assert e.value.code == pkg.ERR_BAD_SHAPE


def test_two_grids_interleaved(pkg, oracle, golden, synth, cfg36):
    cfg, sig = cfg36
    g36 = synth.sea_states(100, seed=9, depth_range=(5.0, 4000.0))
    grid_a = pkg.Snl1Grid(cfg, sig, igrid=41)
    grid_b = pkg.Snl1Grid(golden["cfg"], golden["sig"], igrid=42)
    for _ in range(2):
        s_a, _ = grid_a(g36["a"], g36["cg"], g36["kdmean"])
        s_b, _ = grid_b(golden["a"], golden["cg"], golden["kdmean"])
    assert_bitexact(s_a, oracle.w3snl1(cfg, sig, g36["a"], g36["cg"], g36["kdmean"])[0], "A")
    assert_bitexact(s_b, oracle.w3snl1(golden["cfg"], golden["sig"], golden["a"], golden["cg"],
                                       golden["kdmean"])[0], "B")


def test_full_size_properties(pkg, oracle, synth, cfg36):
    """At the bench's size (262,144 points, 4 GB of traffic per pass): the kernels agree on
    every value, the run is deterministic, and a seeded sample of points equals the oracle."""
    import torch

    cfg, sig = cfg36
    npts = 262144
    g = synth.sea_states_chunked(npts, seed=3, depth_range=(5.0, 4000.0))
    grid = pkg.Snl1Grid(cfg, sig, igrid=6)
    dev = torch.device("cuda:0")
    a = torch.from_numpy(g["a"]).to(dev)
    cg = torch.from_numpy(g["cg"]).to(dev)
    kd = torch.from_numpy(g["kdmean"]).to(dev)
    outs = []
    stream = torch.cuda.current_stream().cuda_stream
    for name in ("band", "band", "pair", "pair-general", "rowshift", "gather"):
        grid.select_kernel(kernel_id(pkg, name))
        s = torch.empty_like(a)
        d = torch.empty_like(a)
        grid.run_device(npts, a, cg, kd, s, d, stream)
        torch.cuda.synchronize()
        outs.append((s.view(torch.int32), d.view(torch.int32)))
    for s_, d_ in outs[1:]:
        assert torch.equal(s_, outs[0][0]) and torch.equal(d_, outs[0][1])
    idx = np.random.default_rng(0).choice(npts, 2000, replace=False)
    s_ref, d_ref = oracle.w3snl1(cfg, sig, g["a"][idx], g["cg"][idx], g["kdmean"][idx])
    assert_bitexact(outs[0][0].view(torch.float32).cpu().numpy()[idx], s_ref, "S sample")
    assert_bitexact(outs[0][1].view(torch.float32).cpu().numpy()[idx], d_ref, "D sample")


def test_autotune_picks_a_kernel_that_stays_bitexact(pkg, oracle, synth, cfg36):
    """ww_snl1_autotune times every kernel the tables fit, selects one, records it in the
    report; the grid then still gives the oracle's bits."""
    cfg, sig = cfg36
    grid = pkg.Snl1Grid(cfg, sig, igrid=7)
    k = pkg.snl1_autotune(7)
    assert k in (pkg.KERNEL_PAIR, pkg.KERNEL_PAIR_GENERAL, pkg.KERNEL_BAND, pkg.KERNEL_TILE,
                 pkg.KERNEL_ROWSHIFT, pkg.KERNEL_GATHER)
    rep = pkg.autotune_report()
    key = next(x for x in rep if x.startswith("dia 36x36"))
    assert rep[key]["choice"] == k and len(rep[key]["ms"]) >= 5
    g = synth.sea_states(300, seed=77, depth_range=(5.0, 4000.0))
    s, d = grid(g["a"], g["cg"], g["kdmean"])
    s_ref, d_ref = oracle.w3snl1(cfg, sig, g["a"], g["cg"], g["kdmean"])
    assert_bitexact(s, s_ref, "S after autotune")
    assert_bitexact(d, d_ref, "D after autotune")


def test_bounded_wait_reports_instead_of_hanging(pkg, oracle, synth, cfg36):
    """The failure path of the DIA's bulk-copy waits, made to run out on purpose: with the test
    hook every CTA expects bytes its first copy never brings; its bounded wait gives up (about a
    second), the launch ends, ww_snl1 reports ERR_KERNEL, and the next call is exact again."""
    import ctypes
    import time

    cfg, sig = cfg36
    grid = pkg.Snl1Grid(cfg, sig, igrid=8)
    grid.select_kernel(pkg.KERNEL_PAIR)
    L = pkg.lib()
    L.ww_snl1_test_stall.argtypes = [ctypes.c_int, ctypes.c_int]
    L.ww_snl1_test_stall.restype = ctypes.c_int
    g = synth.sea_states(600, seed=88, depth_range=(5.0, 4000.0))
    assert L.ww_snl1_test_stall(8, 16) == pkg.OK
    t0 = time.time()
    try:
        grid(g["a"], g["cg"], g["kdmean"])
    except pkg.WwError:
        pass
    assert pkg.last_error() == pkg.ERR_KERNEL
    assert time.time() - t0 < 120
    assert L.ww_snl1_test_stall(8, 0) == pkg.OK
    s, d = grid(g["a"], g["cg"], g["kdmean"])
    assert pkg.last_error() == pkg.OK
    s_ref, d_ref = oracle.w3snl1(cfg, sig, g["a"], g["cg"], g["kdmean"])
    assert_bitexact(s, s_ref, "S after the stalled call")
    assert_bitexact(d, d_ref, "D after the stalled call")
