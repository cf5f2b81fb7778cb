"""A whole time step on the resident VA recorded once and replayed as one CUDA graph
(ww_step_begin / ww_step_end / ww_step_run), against the same calls run one by one on the GPU and
against the reference's own C++ running them on the CPU (oracle/_ref/libref_ww3_scalar.so, its
resident-VA entries): W3KTP3, W3XYP3, W3KTP3 again and W3SRCE with ST4, per step, W3WAVE's order
of the propagation and source-term parts. Two steps; every VA bit must agree."""

import ctypes

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available
import st4_common as sc

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
KTP3_ARRAYS = ("sig", "dsip", "ecos", "esin", "ec2", "esc", "es2", "mapwn", "mapth2", "mapwn2")
XYP3_ARRAYS = ("mapsf", "clats", "sig", "ecos", "esin", "dpdx", "dpdy", "dqdx", "dqdy", "gsqrt",
               "atrnx", "atrny", "mapx2", "mapy2", "mapaxy", "mapcxy", "maptrn", "mapsta", "cg",
               "cx", "cy")


def _bind(L):
    L.ww_ktp3_batch_va.argtypes = [I, P, I, P, I] + [P] * 10 + [I, I, F, F, I, P, P, I, P, P, P,
                                                               P, I, I, P, P]
    L.ww_ktp3_batch_va.restype = I
    L.ww_xyp3_batch_va.argtypes = [I, P, I, P, I, P, I, P, I, F] + [P] * 21 + [
        I, I, P, P, P, P, P, I, I]
    L.ww_xyp3_batch_va.restype = I
    L.ww_srce_batch_va.argtypes = [I, I, I, I, I, F, P, I, I, I] + [P] * 9
    L.ww_srce_batch_va.restype = None
    L.ww_srce_last_error.restype = I
    L.ww_va_host_read.argtypes = [I, P, I, I]
    L.ww_va_host_read.restype = I
    L.ww_va_host_write.argtypes = [I, P, I, I]
    L.ww_va_host_write.restype = I
    if hasattr(L, "ww_wave_cflxy"):
        L.ww_wave_cflxy.argtypes = [I] * 9 + [F, F, F] + [P] * 12
        L.ww_wave_cflxy.restype = I
    return L


class Calls:
    """The four calls of one step on library L, grid igrid, resident VA bound to va."""

    def __init__(self, L, igrid, va, kc, xc, pts):
        self.L, self.ig, self.va = L, igrid, va
        self.kc = {k: np.ascontiguousarray(v) for k, v in kc.items() if isinstance(v, np.ndarray)}
        self.kcs = kc
        self.xc = {k: np.ascontiguousarray(v) for k, v in xc.items() if isinstance(v, np.ndarray)}
        self.xcs = xc
        self.pts = {k: np.array(v, copy=True) for k, v in pts.items()}
        n = va.shape[0] - 1
        self.jsea = np.arange(1, n + 1, dtype=np.int32)
        self.shave = np.zeros(n, np.int32)
        self.cth = np.array(kc["cflthmax"], np.float32, copy=True)
        self.ck = np.array(kc["cflkmax"], np.float32, copy=True)

    def ktp3(self, itstep):
        k, ks, L = self.kc, self.kcs, self.L
        rc = L.ww_ktp3_batch_va(
            self.ig, k["rpar"].ctypes.data, k["rpar"].size, k["ipar"].ctypes.data,
            k["ipar"].size, *[k[a].ctypes.data for a in KTP3_ARRAYS], itstep, 1, ks["facth"],
            ks["fack"], ks["nsea"], k["cg"].ctypes.data, k["wn"].ctypes.data, ks["npts"],
            k["jsea"].ctypes.data, k["isea"].ctypes.data, k["pscal"].ctypes.data,
            self.va.ctypes.data, self.va.shape[1], self.va.shape[0] - 1, self.cth.ctypes.data,
            self.ck.ctypes.data)
        assert rc == 0, rc

    def xyp3(self):
        x, xs, L = self.xc, self.xcs, self.L
        rc = L.ww_xyp3_batch_va(
            self.ig, x["rpar"].ctypes.data, x["rpar"].size, x["ipar"].ctypes.data, x["ipar"].size,
            x["imaps"].ctypes.data, x["imaps"].size, x["tscal"].ctypes.data, x["tscal"].size,
            xs["dtg"], *[x[a].ctypes.data for a in XYP3_ARRAYS], xs["flbpi"], xs["nbi"],
            x["isbpi"].ctypes.data, x["bbpi0"].ctypes.data, x["bbpin"].ctypes.data,
            x["on"].ctypes.data, self.va.ctypes.data, self.va.shape[1], self.va.shape[0] - 1)
        assert rc == 0, rc

    def srce(self):
        p, L = self.pts, self.L
        n = self.va.shape[0] - 1
        L.ww_srce_batch_va(self.ig, 1, 0, 1, 1, 900.0, self.va.ctypes.data, self.va.shape[1], n,
                           n, self.jsea.ctypes.data, sc.p(p["wn1"]), sc.p(p["cg1"]),
                           sc.p(p["pin"]), sc.p(p["psc"]), sc.p(p["whitecap"]),
                           sc.p(p["taubbl"]), sc.p(p["tauice"]), self.shave.ctypes.data)
        assert L.ww_srce_last_error() == 0

    def cflxy(self):
        """W3CFLXY, W3WAVE's CFL diagnostic before the propagation (wave_w3wave.hpp:548-574)."""
        x, xs = self.xc, self.xcs
        ip = x["ipar"]  # NX, NY, NSEA, NK, NTH, NSPEC, ICLOSE, FLCX, FLCY, FLAGLL, FLCUR
        nsea = int(ip[2])
        self.cfl = np.zeros(nsea, np.float32)
        rc = self.L.ww_wave_cflxy(self.ig, nsea, nsea, int(ip[0]), int(ip[1]), int(ip[3]),
                                  int(ip[4]), int(ip[10]), 0, xs["dtg"], 0.0, 0.0,
                                  *[x[a].ctypes.data for a in ("mapsf", "clats", "ecos", "esin",
                                                               "dpdx", "dpdy", "dqdx", "dqdy",
                                                               "cg", "cx", "cy")],
                                  self.cfl.ctypes.data)
        assert rc == 0, rc

    def step(self, cflxy=False):
        if cflxy:
            self.cflxy()
        self.ktp3(1)
        self.xyp3()
        self.ktp3(2)
        self.srce()

    def read(self):
        assert self.L.ww_va_host_read(self.ig, self.va.ctypes.data, self.va.shape[1],
                                      self.va.shape[0] - 1) == 0
        return self.va


@pytest.fixture(scope="module")
def case(oracle, synth):
    st = synth.st4_setup(variant="default")
    t = oracle.st4_tables(st)
    sr = synth.srce_setup(st)
    xc = synth.xyp3_case(24, 18, seed=41, ref=oracle.ref_w3map3)
    nsea = xc["nsea"]
    kc = synth.ktp3_case(nsea, seed=42, nsea=nsea)
    pts = synth.srce_points(nsea, seed=43)
    return st, t, sr, xc, kc, pts


def _gpu_grid(pkg, oracle, synth, st, t, sr, igrid):
    L = pkg.lib()
    pkg.init()
    rc = oracle.register_st4(lambda *a: L.ww_st4_init(igrid, *a),
                             lambda *a: L.ww_st4_set_real(igrid, *a),
                             lambda *a: L.ww_st4_set_int(igrid, *a),
                             lambda: L.ww_st4_commit(igrid), st, t)
    assert rc == 0
    cfg, sig = synth.dia_config()
    pkg.Snl1Grid(cfg, sig, igrid=igrid)
    rc = L.ww_srce_init(igrid, sc.p(sr["rpar"]), len(sr["rpar"]), sc.p(sr["ipar"]),
                        len(sr["ipar"]), sc.p(sr["sig"]), sc.p(sr["dden"]), sc.p(sr["ecos"]),
                        sc.p(sr["esin"]), sc.p(sr["mapwn"]))
    assert rc == 0
    return _bind(L)


def test_step_graph_equals_calls_and_reference(pkg, oracle, synth, case):
    st, t, sr, xc, kc, pts = case
    nsteps = 2
    # the reference, one call after another on its resident VA (host memory)
    ref = oracle.RefSt4(st, t, igrid=701, srce=sr, dia=synth.dia_config(), scalar_mvec=True)
    R = _bind(ref.L)
    c_ref = Calls(R, 701, np.array(xc["va"], np.float32, copy=True), kc, xc, pts)
    for _ in range(nsteps):
        c_ref.step()
    va_ref = c_ref.read()
    # the library, one call after another
    L = _gpu_grid(pkg, oracle, synth, st, t, sr, 702)
    c_run = Calls(L, 702, np.array(xc["va"], np.float32, copy=True), kc, xc, pts)
    for _ in range(nsteps):
        c_run.step()
    va_run = c_run.read()
    assert_bitexact(va_run, va_ref, "VA, calls on the GPU vs the reference")
    # the library, the step recorded once and replayed as one graph
    _gpu_grid(pkg, oracle, synth, st, t, sr, 703)
    c_rec = Calls(L, 703, np.array(xc["va"], np.float32, copy=True), kc, xc, pts)
    with pkg.Step(703) as step:
        c_rec.step(cflxy=True)
    assert step.ops() == 5
    step.run(nsteps)
    va_rec = c_rec.read()
    assert_bitexact(va_rec, va_ref, "VA, replayed graph vs the reference")
    # the host takes the VA back and rewrites it (ww_va_host_write): the next replay uploads it
    va0 = np.array(xc["va"], np.float32)
    for calls in (c_ref, c_rec):
        assert calls.L.ww_va_host_write(calls.ig, calls.va.ctypes.data, calls.va.shape[1],
                                        calls.va.shape[0] - 1) == 0
        calls.va[...] = va0
    c_ref.step()
    step.run(1)
    assert_bitexact(c_rec.read(), c_ref.read(), "VA, replay after a host write vs the reference")
    step.free()


def test_step_protocol(pkg):
    L = pkg.lib()
    pkg.init()
    step = pkg.Step(709)
    for name in ("ww_step_end", "ww_step_free", "ww_step_ops"):
        getattr(L, name).argtypes = [I]
        getattr(L, name).restype = I
    assert L.ww_step_end(709) == 2  # not recording
    with pytest.raises(pkg.WwError):
        step.run(1)  # nothing recorded
    with step:
        pass
    assert step.ops() == 0
    step.run(3)  # an empty step replays nothing
    step.free()


def test_steps_run_grids_side_by_side(pkg, oracle, synth):
    """Three grids of different sizes, each with its own recorded step: ww_steps_run replays
    them in one call and gives every grid the VA that its
    own ww_step_run gives."""
    st = synth.st4_setup(variant="default")
    t = oracle.st4_tables(st)
    sr = synth.srce_setup(st)
    cases = []
    for nx, ny, seed in [(24, 18, 51), (40, 22, 52), (16, 12, 53)]:
        xc = synth.xyp3_case(nx, ny, seed=seed, ref=oracle.ref_w3map3)
        nsea = xc["nsea"]
        cases.append((xc, synth.ktp3_case(nsea, seed=seed + 1, nsea=nsea),
                      synth.srce_points(nsea, seed=seed + 2)))

    def record(base):
        calls, steps = [], []
        for k, (xc, kc, pts) in enumerate(cases):
            ig = base + k
            L = _gpu_grid(pkg, oracle, synth, st, t, sr, ig)
            c = Calls(L, ig, np.array(xc["va"], np.float32, copy=True), kc, xc, pts)
            step = pkg.Step(ig)
            with step:
                c.step()
            calls.append(c)
            steps.append(step)
        return calls, steps

    sep_calls, sep_steps = record(720)
    for s in sep_steps:
        s.run(2)
    va_sep = [np.array(c.read(), copy=True) for c in sep_calls]
    com_calls, com_steps = record(730)
    pkg.steps_run([730, 731, 732], 2)
    va_com = [np.array(c.read(), copy=True) for c in com_calls]
    for k in range(3):
        assert_bitexact(va_com[k], va_sep[k], f"grid {k}: ww_steps_run vs ww_step_run")
        assert not np.array_equal(va_com[k], cases[k][0]["va"])
    with pytest.raises(pkg.WwError):
        pkg.steps_run([730, 730], 1)  # a grid listed twice
    # The same steps fused: every grid's propagation, then one W3SRCE launch over all 3 grids'
    # points with one work queue; bit-equal to the grids' own graphs.
    fus_calls, fus_steps = record(740)
    pkg.steps_fuse([740, 741, 742])
    pkg.steps_run([740, 741, 742], 2)
    va_fus = [np.array(c.read(), copy=True) for c in fus_calls]
    for k in range(3):
        assert_bitexact(va_fus[k], va_sep[k], f"grid {k}: fused W3SRCE launch vs ww_step_run")
    with pytest.raises(pkg.WwError):
        pkg.steps_fuse([740, 740])  # a grid listed twice
    with pytest.raises(pkg.WwError):
        pkg.steps_fuse([740, 799])  # a grid with no recorded step
    pkg.steps_fuse([])
    for s in sep_steps + com_steps + fus_steps:
        s.free()
