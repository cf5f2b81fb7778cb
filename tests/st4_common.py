"""Shared driving code of the ST4 / W3SRCE tests: one backend interface over the reference's
build (oracle/_ref), the host build of the kernels' source (tests/hemu.cpp) and the CUDA library,
all with the reference's C ABI argument lists."""

import ctypes
import pathlib
import subprocess

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
NK_ARGS = ("xfr", "dth", "lam", "snlc1", "kdcon", "kdmn", "snls1", "snls2", "snls3", "fachfe")


def p(x):
    return None if x is None else x.ctypes.data


def build_hemu(out_dir):
    """Compile tests/hemu.cpp with the kernels' headers for the host; returns the CDLL."""
    so = pathlib.Path(out_dir) / "libhemu.so"
    csrc = ROOT / "ww3-gpu_b200" / "csrc"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-math-errno",
                    "-fPIC", "-shared", f"-I{csrc}", "-I/usr/local/cuda/include",
                    str(ROOT / "tests" / "hemu.cpp"), str(csrc / "snl1_tables.cpp"), "-o",
                    str(so)], check=True)
    H = ctypes.CDLL(str(so))
    H.hemu_st4_init.argtypes = [P, I, P, I]
    H.hemu_st4_set_real.argtypes = [I, P, I, P, P]
    H.hemu_st4_set_int.argtypes = [I, P, I, P, P]
    H.hemu_sds4.argtypes = [I] + [P] * 8 + [I, I] + [P] * 4
    H.hemu_sin4.argtypes = [I] + [P] * 17
    H.hemu_spr4.argtypes = [I] + [P] * 20
    H.hemu_snl1_init.argtypes = [I, I] + [F] * 10 + [P]
    H.hemu_srce_init.argtypes = [P, I, P, I, P, P, P, P, P]
    H.hemu_srce_batch.argtypes = [I, I, I, I, F, I] + [P] * 9
    return H


class Backend:
    """ST4 / W3SRCE calls of one implementation. ``fn(name)`` gives the entry with the
    reference's argument list minus igrid."""

    def __init__(self, fn, last_error=None):
        self.fn = fn
        self.last_error = last_error

    def sds4(self, a, k, cg, ustar, usdir, depth, dair, dlw, f57=1, f58=1):
        n = a.shape[0]
        srhs, ddiag, brl = np.zeros_like(a), np.zeros_like(a), np.zeros_like(a)
        wc = np.zeros((n, 4), np.float32)
        self.fn("sds4")(n, p(a), p(k), p(cg), p(ustar), p(usdir), p(depth), p(dair), p(dlw),
                        f57, f58, p(srhs), p(ddiag), p(brl), p(wc))
        return {"srhs": srhs, "ddiag": ddiag, "brlambda": brl, "whitecap": wc}

    def sin4(self, a, cg, k, u, ustar, drat, as_, usdir, z0, cd, tauwx, tauwy):
        n = a.shape[0]
        tx, ty = tauwx.copy(), tauwy.copy()
        tnx, tny = np.zeros(n, np.float32), np.zeros(n, np.float32)
        s, d = np.zeros_like(a), np.zeros_like(a)
        llws = np.zeros(a.shape, np.int32)
        self.fn("sin4")(n, p(a), p(cg), p(k), p(u), p(ustar), p(drat), p(as_), p(usdir), p(z0),
                        p(cd), p(tx), p(ty), p(tnx), p(tny), p(s), p(d), p(llws))
        return {"s": s, "d": d, "llws": llws, "tauwx": tx, "tauwy": ty, "tauwnx": tnx,
                "tauwny": tny}

    def spr4(self, a, cg, wn, u, udir, tauwx, tauwy, llws, ustar, usdir):
        n = a.shape[0]
        us, ud = ustar.copy(), usdir.copy()
        names = ("emean", "fmean", "fmean1", "wnmean", "amax", "cd", "z0", "charn", "fmeanws",
                 "dlwmean")
        outs = [np.zeros(n, np.float32) for _ in names]
        self.fn("spr4")(n, p(a), p(cg), p(wn), p(u), p(udir), p(tauwx), p(tauwy), p(llws),
                        p(us), p(ud), *[p(o) for o in outs])
        r = dict(zip(names, outs))
        r["ustar"], r["usdir"] = us, ud
        return r

    def srce_batch(self, pts, it=1, inflags24=0, f57=1, f58=1, dtg=900.0):
        n = pts["spec"].shape[0]
        r = {k: pts[k].copy() for k in ("spec", "psc", "whitecap", "taubbl", "tauice")}
        r["shave"] = np.zeros(n, np.int32)
        self.fn("srce_batch")(it, inflags24, f57, f58, dtg, n, p(r["spec"]), p(pts["wn1"]),
                              p(pts["cg1"]), p(pts["pin"]), p(r["psc"]), p(r["whitecap"]),
                              p(r["taubbl"]), p(r["tauice"]), p(r["shave"]))
        return r


def hemu_backend(H):
    return Backend(lambda name: getattr(H, "hemu_" + name))


def ref_backend(L, igrid):
    return Backend(lambda name: (lambda *a: getattr(L, "ww_" + name)(igrid, *a)),
                   lambda: L.ww_srce_last_error())


def setup_hemu(H, oracle, st, t, srce=None, dia=None):
    rc = oracle.register_st4(H.hemu_st4_init, H.hemu_st4_set_real, H.hemu_st4_set_int,
                             H.hemu_st4_commit, st, t)
    assert rc == 0
    if dia is not None:
        cfg, sig = dia
        assert H.hemu_snl1_init(cfg["nk"], cfg["nth"], *[cfg[k] for k in NK_ARGS], p(sig)) == 0
    if srce is not None:
        assert H.hemu_srce_init(p(srce["rpar"]), len(srce["rpar"]), p(srce["ipar"]),
                                len(srce["ipar"]), p(srce["sig"]), p(srce["dden"]),
                                p(srce["ecos"]), p(srce["esin"]), p(srce["mapwn"])) == 0


def point_inputs(pts):
    """The per-point ST4 call arguments the tests use, from synth.srce_points."""
    n, nth = pts["spec"].shape[0], pts["spec"].shape[1] // pts["wn1"].shape[1]
    psc, pin = pts["psc"], pts["pin"]
    return {
        "a": pts["spec"], "k": pts["wn1"], "cg": pts["cg1"],
        "k2": np.repeat(pts["wn1"], nth, axis=1).astype(np.float32),
        "ustar": psc[:, 0].copy(), "usdir": psc[:, 1].copy(), "depth": pin[:, 0].copy(),
        "dair": pin[:, 5].copy(), "dlw": (0.9 * psc[:, 1]).astype(np.float32),
        "u": pin[:, 1].copy(), "drat": (pin[:, 5] / np.float32(1000.0)).astype(np.float32),
        "as": np.zeros(n, np.float32), "z0": np.full(n, 1e-4, np.float32),
        "cd": np.full(n, 1.2e-3, np.float32), "tauwx": psc[:, 2].copy(),
        "tauwy": psc[:, 3].copy(),
    }


def run_all(be, x, llws=None):
    """SDS4, SIN4 and SPR4 of every point through one backend."""
    out = {"sds4": be.sds4(x["a"], x["k"], x["cg"], x["ustar"], x["usdir"], x["depth"], x["dair"],
                           x["dlw"]),
           "sin4": be.sin4(x["a"], x["cg"], x["k2"], x["u"], x["ustar"], x["drat"], x["as"],
                           x["usdir"], x["z0"], x["cd"], x["tauwx"], x["tauwy"])}
    lw = out["sin4"]["llws"] if llws is None else llws
    out["spr4"] = be.spr4(x["a"], x["cg"], x["k"], x["u"], x["usdir"], x["tauwx"], x["tauwy"],
                          lw, x["ustar"], x["usdir"])
    return out
