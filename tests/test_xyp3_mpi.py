"""W3XYP3 under W3_MPI: ww_xyp3_batch_mpi, ww_xyp3_mpi_pack/unpack and the exchange around them.

Property (size-independent): with the sea points split over NAPROC ranks and the spectral
components over the same ranks (any IAPPRO), pack -> exchange -> ww_xyp3_batch_mpi -> exchange
-> unpack leaves every rank's columns equal, bit for bit, to the same columns of one W3_SHRD
ww_xyp3_batch over the whole grid: every value is copied, never combined (the reference's
PATCH.md:2472-2490). The checker of the single-rank step is the reference's own C++
(oracle/_ref/libref_ww3.so), which also exports the MPI entries, so its ww_xyp3_batch_mpi is
compared with the library's directly as well.

The multi-rank host logic (ww3_gpu_b200.xyp3_mpi: the message layout and the two exchanges) runs
as world_size 2 and 3 gloo ranks on the CPU, each rank's compute being the reference build; on
a GPU the library's entries run for every rank, the ranks emulated in one process one after
another (nothing waits on another rank inside a kernel).
"""

import ctypes
import importlib
import os
import socket

import numpy as np
import pytest

from conftest import assert_bitexact, cuda_available
from oracle import oracle as _oracle

needs_ref = pytest.mark.skipif(not _oracle.ref_available(), reason="oracle/_ref not built")

SMALL = dict(nx=23, ny=17, nk=6, nth=8)


def _mpi_mod():
    import __graft_entry__ as entry

    entry.load_package()
    return importlib.import_module("ww3_gpu_b200.xyp3_mpi")


def _ref_bound():
    L = _oracle.ref_lib()
    m = _mpi_mod()
    m.bind(L)
    P, I = ctypes.c_void_p, ctypes.c_int
    L.ww_va_host_read.argtypes = [I, P, I, I]
    L.ww_va_host_read.restype = I
    return L


def _iappro(nspec, naproc, seed):
    rng = np.random.default_rng(seed)
    own = rng.integers(1, naproc + 1, nspec).astype(np.int32)
    own[:naproc] = np.arange(1, naproc + 1)  # every rank owns at least one component
    return own


# ------------------------------------------------------------------ host logic, no library
def test_columns_roundtrip_and_layout():
    m = _mpi_mod()
    rng = np.random.default_rng(0)
    for nsea, naproc in ((17, 1), (17, 2), (17, 3), (40, 4), (5, 8)):
        va = rng.random((nsea + 1, 12), dtype=np.float32)
        nsealm = m.nsealm_of(nsea, naproc)
        loc = [m.local_columns(va, naproc, ip, nsealm) for ip in range(1, naproc + 1)]
        back = m.global_columns(loc, nsea)
        assert np.array_equal(back[1:], va[1:])
        iappro = _iappro(12, naproc, 1) if naproc <= 12 else None
        for ip in range(1, naproc + 1):
            lay = m.layout(iappro, naproc, ip, nsea)
            assert lay.nbuf == sum(lay.recv_counts) == (naproc - 1) * len(lay.own) * nsealm
            assert sum(lay.send_counts) == len(lay.pack_isps) * nsealm
            offs = [lay.poff[j - 1] for j in range(1, naproc + 1) if j != ip]
            assert offs == sorted(offs) and (not offs or offs[0] == 0)
            # what rank ip sends to rank j is what j expects from ip
            for j in range(1, naproc + 1):
                if j != ip:
                    other = m.layout(iappro, naproc, j, nsea)
                    assert lay.send_counts[j - 1] == other.recv_counts[ip - 1]


# ------------------------------------------------------------------ gloo ranks, reference compute
def _gloo_rank(rank, world, port, case_kw, seed, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import __graft_entry__ as entry

        entry.load_package()
        synth = importlib.import_module("ww3_gpu_b200.synth")
        m = _mpi_mod()
        L = _ref_bound()
        c = synth.xyp3_case(ref=_oracle.ref_w3map3, seed=seed, **case_kw)
        nsealm = m.nsealm_of(c["nsea"], world)
        va = m.local_columns(c["va"], world, rank + 1, nsealm)
        igrid = 40 + rank
        rc = m.step_dist(L, igrid, c, va, _iappro(va.shape[1], world, seed))
        assert rc == 0, rc
        assert L.ww_va_host_read(igrid, va.ctypes.data, va.shape[1], nsealm) == 0
        np.save(out % rank, va)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@needs_ref
@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_equal_single_rank(world, tmp_path):
    import torch.multiprocessing as mp

    m = _mpi_mod()
    import __graft_entry__ as entry

    entry.load_package()
    synth = importlib.import_module("ww3_gpu_b200.synth")
    kw = dict(SMALL, iclose=2, flcur=True, flbpi=True)
    seed = 11 + world
    c = synth.xyp3_case(ref=_oracle.ref_w3map3, seed=seed, **kw)
    rc, va_ref = _oracle.xyp3_call(_oracle.ref_lib(), c)
    assert rc == 0
    out = str(tmp_path / "va_%d.npy")
    mp.start_processes(_gloo_rank, args=(world, _free_port(), kw, seed, out), nprocs=world,
                       start_method="spawn")
    loc = [np.load(out % r) for r in range(world)]
    got = m.global_columns(loc, c["nsea"])
    assert_bitexact(got[1:], va_ref[1:], f"VA after {world}-rank W3XYP3")


# ------------------------------------------------------------------ the library on a GPU
@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("world,case", [
    (2, dict(nx=48, ny=32, iclose=2, flcur=True, flbpi=True)),
    (3, dict(nx=37, ny=29, iclose=-1, flcur=False, flbpi=True, nk=12, nth=24)),
])
def test_mpi_ranks_equal_single_rank_gpu(pkg, synth, world, case):
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    m = _mpi_mod()
    L = m.bind(pkg.lib())
    pkg.init()
    seed = 21 + world
    c = synth.xyp3_case(ref=_oracle.ref_w3map3, seed=seed, **case)
    rc, va_ref = _oracle.xyp3_call(_oracle.ref_lib(), c)
    assert rc == 0
    nsealm = m.nsealm_of(c["nsea"], world)
    vas = [m.local_columns(c["va"], world, ip, nsealm) for ip in range(1, world + 1)]
    igrids = [300 + 10 * world + ip for ip in range(1, world + 1)]  # one VA per grid
    rcs = m.step_local(L, igrids, c, vas, _iappro(vas[0].shape[1], world, seed))
    assert rcs == [0] * world
    for g, v in zip(igrids, vas):
        assert pkg.va_host_read(g, v) == 0
    assert_bitexact(m.global_columns(vas, c["nsea"])[1:], va_ref[1:],
                    f"VA after {world}-rank W3XYP3 (B200)")


@needs_ref
@pytest.mark.gpu
def test_batch_mpi_matches_reference_entry(pkg, synth):
    """One rank's ww_xyp3_batch_mpi (VA and the send-back buffer) against the reference's."""
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    m = _mpi_mod()
    L = m.bind(pkg.lib())
    pkg.init()
    R = _ref_bound()
    world, me = 3, 2
    c = synth.xyp3_case(ref=_oracle.ref_w3map3, seed=5, nx=40, ny=24, iclose=2, flcur=True,
                        flbpi=True)
    nsealm = m.nsealm_of(c["nsea"], world)
    lay = m.layout(_iappro(c["va"].shape[1], world, 5), world, me, c["nsea"])
    rng = np.random.default_rng(9)
    rbuf = rng.random(lay.nbuf, dtype=np.float32) * np.float32(1e-3)
    outs = []
    for lib_, igrid, host_read in ((L, 401, pkg.va_host_read), (R, 402, None)):
        va = m.local_columns(c["va"], world, me, nsealm)
        rc, sbuf = m.propagate(lib_, igrid, c, va, lay, rbuf)
        assert rc == 0
        if host_read is not None:
            assert host_read(igrid, va) == 0
        else:
            assert R.ww_va_host_read(igrid, va.ctypes.data, va.shape[1], nsealm) == 0
        outs.append((va, sbuf))
    assert_bitexact(outs[0][0], outs[1][0], "this rank's VA")
    assert_bitexact(outs[0][1], outs[1][1], "SSTORE blocks")


@needs_ref
@pytest.mark.gpu
def test_batch_mpi_validation(pkg, synth):
    if not cuda_available():
        pytest.skip("needs a CUDA device")
    m = _mpi_mod()
    L = m.bind(pkg.lib())
    pkg.init()
    c = synth.xyp3_case(ref=_oracle.ref_w3map3, seed=6, **SMALL)
    world = 2
    nsealm = m.nsealm_of(c["nsea"], world)
    lay = m.layout(_iappro(c["va"].shape[1], world, 6), world, 1, c["nsea"])
    va = m.local_columns(c["va"], world, 1, nsealm)
    before = va.copy()
    rbuf = np.zeros(lay.nbuf, np.float32)
    bad = m.Layout(**{**lay.__dict__, "poff": lay.poff + 1})  # rank 2's block not at 0
    rc, _ = m.propagate(L, 501, c, va, bad, rbuf)
    assert rc == 2 and np.array_equal(va, before)
    bad = m.Layout(**{**lay.__dict__, "iaproc": 3})  # IAPROC > NAPROC
    rc, _ = m.propagate(L, 501, c, va, bad, rbuf)
    assert rc == 2
    isps = np.array([0], np.int32)  # a component outside VA
    buf = np.zeros(nsealm, np.float32)
    assert L.ww_xyp3_mpi_pack(501, va.ctypes.data, va.shape[1], nsealm, isps.ctypes.data, 1,
                              buf.ctypes.data) == 2
