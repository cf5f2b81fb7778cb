"""ww_snl1_noalloc, the W3SNL1 entry that allocates no device memory, through the C ABI.

It stages through a static device array instead of per-grid buffers and launches the same
kernel as ww_snl1, so its S and D equal ww_snl1's bit for bit (float32, same operation order);
two calls in a row must both match, and the device's free memory must not move across them.
The file is named to be collected last, so the test also runs after every other GPU test; it
passes alone in a fresh process as well (its own init, its own grid number).
"""

import ctypes

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

IGRID = 77
STATIC_FLOATS = 8 << 20


def _p(x):
    return ctypes.c_void_p(x.ctypes.data)


def max_points(nspec, nk):
    c = lambda n: (n + 63) // 64 * 64  # noqa: E731
    n = STATIC_FLOATS // (3 * nspec + nk + 1)
    while 3 * c(n * nspec) + c(n * nk) + c(n) > STATIC_FLOATS:
        n -= 1
    return n


def test_noalloc_matches_host_entry_twice(pkg, synth):
    import torch

    L = pkg.lib()
    cfg, sig = synth.dia_config()
    grid = pkg.Snl1Grid(cfg, sig, igrid=IGRID)
    npts = 1500
    g = synth.sea_states(npts, seed=4242, depth_range=(5.0, 4000.0))
    s_ref, d_ref = grid(g["a"], g["cg"], g["kdmean"])  # ww_snl1, the existing entry
    # Free device memory before the first call: the set-up of that call (resolving the static
    # array's address) must not allocate either. The DIA kernel's module, which holds the
    # array, is already loaded by the ww_snl1 call above.
    torch.cuda.mem_get_info(0)
    free_before = torch.cuda.mem_get_info(0)[0]

    a, cg, kd = g["a"], g["cg"], g["kdmean"]
    for call in range(2):
        s = np.full_like(a, np.nan)
        d = np.full_like(a, np.nan)
        L.ww_snl1_noalloc(IGRID, npts, _p(a), _p(cg), _p(kd), _p(s), _p(d))
        assert pkg.last_error() == pkg.OK, f"call {call}"
        assert_bitexact(s, s_ref, f"S, call {call}")
        assert_bitexact(d, d_ref, f"D, call {call}")
        assert torch.cuda.mem_get_info(0)[0] == free_before, (
            f"device memory moved across ww_snl1_noalloc call {call}")


def test_noalloc_size_limit(pkg, synth):
    L = pkg.lib()
    cfg, sig = synth.dia_config()
    grid = pkg.Snl1Grid(cfg, sig, igrid=IGRID + 1)
    nspec, nk = grid.nspec, grid.nk
    most = max_points(nspec, nk)
    assert most == 2137  # 36x36
    g = synth.sea_states(most + 1, seed=99, depth_range=(5.0, 4000.0))
    s = np.full_like(g["a"], 7.0)
    d = np.full_like(g["a"], 7.0)
    L.ww_snl1_noalloc(IGRID + 1, most + 1, _p(g["a"]), _p(g["cg"]), _p(g["kdmean"]), _p(s), _p(d))
    assert pkg.last_error() == pkg.ERR_BAD_SHAPE
    assert np.all(s == 7.0) and np.all(d == 7.0)
    # The largest batch that fits runs and matches ww_snl1.
    a, cg, kd = g["a"][:most], g["cg"][:most], g["kdmean"][:most]
    s_ref, d_ref = grid(a, cg, kd)
    s = np.empty_like(a)
    d = np.empty_like(a)
    L.ww_snl1_noalloc(IGRID + 1, most, _p(a), _p(cg), _p(kd), _p(s), _p(d))
    assert pkg.last_error() == pkg.OK
    assert_bitexact(s, s_ref, "S at the limit")
    assert_bitexact(d, d_ref, "D at the limit")
