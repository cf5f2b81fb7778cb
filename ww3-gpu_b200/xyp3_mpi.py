"""W3XYP3 under W3_MPI: the exchange around ww_xyp3_batch_mpi, for a host driver in Python.

WAVEWATCH III's MPI build splits the sea points over ranks (sea point ISEA is column
K = (ISEA-1)/NAPROC + 1 of rank IP = MOD(ISEA-1,NAPROC) + 1) and the spectral components too
(IAPPRO(ISPEC) names the rank that propagates ISPEC). One propagation step on rank IAPROC, as
the WW3 fork's W3KOKKOS_XYP3 runs it (reference: kokkos/src/fortran_iface/PATCH.md:2442-2470,
prop3_c.hpp:48-70):

1. ``ww_xyp3_mpi_pack``: for every other rank IP in rank order and every component IP owns,
   ascending, VA(ISP, 1:NSEALM) of this rank into one send buffer;
2. one message per rank pair (here ``torch.distributed.all_to_all_single``, or an in-process
   exchange when the ranks are emulated in one process);
3. ``ww_xyp3_batch_mpi`` on this rank's components, reading the other ranks' sea points from
   the received blocks and writing W3SCAT's values for them into the send-back blocks;
4. the transposed messages;
5. ``ww_xyp3_mpi_unpack``: the components other ranks own, into this rank's VA.

Every value is copied, never combined, so the bits equal a single-rank (W3_SHRD) step.
The library ``L`` is any handle that exports the three entries with the reference's C ABI
(``ctypes.CDLL`` of libww_b200.so).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

_F, _I, _P = ctypes.c_float, ctypes.c_int, ctypes.c_void_p

XYP3_ARRAYS = ("mapsf", "clats", "sig", "ecos", "esin", "dpdx", "dpdy", "dqdx", "dqdy", "gsqrt",
               "atrnx", "atrny", "mapx2", "mapy2", "mapaxy", "mapcxy", "maptrn", "mapsta", "cg",
               "cx", "cy")


def nsealm_of(nsea: int, naproc: int) -> int:
    """NSEALM: the most sea points a rank holds, CEILING(NSEA/NAPROC)."""
    return (nsea + naproc - 1) // naproc


def local_columns(va_global: np.ndarray, naproc: int, iaproc: int, nsealm: int) -> np.ndarray:
    """Rank iaproc's VA(NSPEC, 0:NSEALM) (numpy shape (NSEALM+1, NSPEC)) cut from a W3_SHRD
    VA(NSPEC, 0:NSEA): column K holds ISEA = IAPROC + (K-1)*NAPROC, 0 past NSEA."""
    nsea = va_global.shape[0] - 1
    out = np.zeros((nsealm + 1, va_global.shape[1]), np.float32)
    isea = iaproc + naproc * np.arange(nsealm)
    ok = isea <= nsea
    out[1:][ok] = va_global[isea[ok]]
    return out


def global_columns(locals_: list, nsea: int) -> np.ndarray:
    """The inverse of local_columns over all ranks (column 0 taken from rank 1)."""
    naproc = len(locals_)
    out = np.zeros((nsea + 1, locals_[0].shape[1]), np.float32)
    out[0] = locals_[0][0]
    for ip, v in enumerate(locals_, start=1):
        isea = ip + naproc * np.arange(v.shape[0] - 1)
        ok = isea <= nsea
        out[isea[ok]] = v[1:][ok]
    return out


@dataclass
class Layout:
    """The message layout of one rank for one ownership IAPPRO (1-based rank per component)."""

    naproc: int
    iaproc: int
    nsealm: int
    own: np.ndarray         # this rank's components, ascending (1-based)
    others: list            # others[IP-1]: the components rank IP owns, ascending
    pack_isps: np.ndarray   # the components other ranks own, by rank then ascending
    send_counts: list       # step 2: values to rank IP (VA of its components)
    recv_counts: list       # step 2: values from rank IP (its VA of this rank's components)
    poff: np.ndarray        # offset of rank IP's block in rbuf and sbuf (rank order)

    @property
    def nbuf(self) -> int:
        return (self.naproc - 1) * len(self.own) * self.nsealm


def layout(iappro, naproc: int, iaproc: int, nsea: int) -> Layout:
    iappro = np.asarray(iappro)
    if iappro.min() < 1 or iappro.max() > naproc:
        raise ValueError("IAPPRO names a rank outside 1..NAPROC")
    nsealm = nsealm_of(nsea, naproc)
    comps = [np.flatnonzero(iappro == ip).astype(np.int32) + 1 for ip in range(1, naproc + 1)]
    own = comps[iaproc - 1]
    pack = [comps[ip - 1] for ip in range(1, naproc + 1) if ip != iaproc]
    pack_isps = np.concatenate(pack).astype(np.int32) if pack else np.zeros(0, np.int32)
    send = [0 if ip == iaproc else len(comps[ip - 1]) * nsealm for ip in range(1, naproc + 1)]
    recv = [0 if ip == iaproc else len(own) * nsealm for ip in range(1, naproc + 1)]
    poff = np.zeros(naproc, np.int32)
    off = 0
    for ip in range(1, naproc + 1):
        if ip == iaproc:
            continue
        poff[ip - 1] = off
        off += len(own) * nsealm
    return Layout(naproc, iaproc, nsealm, own, comps, pack_isps, send, recv, poff)


def bind(L):
    """Declares the three entries' signatures on the ctypes handle L."""
    L.ww_xyp3_batch_mpi.argtypes = ([_I, _P, _I, _P, _I, _P, _I, _P, _I, _F] + [_P] * 21 +
                                    [_I, _I, _P, _P, _P, _P, _P, _I, _I, _I, _I, _P, _P, _P, _I])
    L.ww_xyp3_batch_mpi.restype = _I
    L.ww_xyp3_mpi_pack.argtypes = [_I, _P, _I, _I, _P, _I, _P]
    L.ww_xyp3_mpi_pack.restype = _I
    L.ww_xyp3_mpi_unpack.argtypes = [_I, _P, _I, _I, _P, _I, _P]
    L.ww_xyp3_mpi_unpack.restype = _I
    return L


def pack(L, igrid, va, lay: Layout) -> np.ndarray:
    """Step 1: the send buffer of step 2 (VA of the other ranks' components)."""
    buf = np.zeros(len(lay.pack_isps) * lay.nsealm, np.float32)
    rc = L.ww_xyp3_mpi_pack(igrid, va.ctypes.data, va.shape[1], lay.nsealm,
                            lay.pack_isps.ctypes.data, len(lay.pack_isps), buf.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ww_xyp3_mpi_pack: status {rc}")
    return buf


def unpack(L, igrid, va, lay: Layout, buf: np.ndarray) -> None:
    """Step 5: the other ranks' components of this rank's points, into VA."""
    buf = np.ascontiguousarray(buf, np.float32)
    rc = L.ww_xyp3_mpi_unpack(igrid, va.ctypes.data, va.shape[1], lay.nsealm,
                              lay.pack_isps.ctypes.data, len(lay.pack_isps), buf.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ww_xyp3_mpi_unpack: status {rc}")


def propagate(L, igrid, case, va, lay: Layout, rbuf: np.ndarray):
    """Step 3: ww_xyp3_batch_mpi on this rank's components. Returns (status, sbuf)."""
    nspec = va.shape[1]
    on = np.zeros(nspec, np.int32)
    on[lay.own - 1] = 1
    keep = {k: np.ascontiguousarray(case[k]) for k in
            ("rpar", "ipar", "imaps", "tscal", "isbpi", "bbpi0", "bbpin") + XYP3_ARRAYS}
    rbuf = np.ascontiguousarray(rbuf, np.float32)
    sbuf = np.full(lay.nbuf, np.nan, np.float32)
    rc = L.ww_xyp3_batch_mpi(
        igrid, keep["rpar"].ctypes.data, keep["rpar"].size, keep["ipar"].ctypes.data,
        keep["ipar"].size, keep["imaps"].ctypes.data, keep["imaps"].size,
        keep["tscal"].ctypes.data, keep["tscal"].size, case["dtg"],
        *[keep[k].ctypes.data for k in XYP3_ARRAYS], case["flbpi"], case["nbi"],
        keep["isbpi"].ctypes.data, keep["bbpi0"].ctypes.data, keep["bbpin"].ctypes.data,
        on.ctypes.data, va.ctypes.data, nspec, lay.nsealm, lay.naproc, lay.iaproc,
        lay.poff.ctypes.data, rbuf.ctypes.data, sbuf.ctypes.data, lay.nbuf)
    return rc, sbuf


def _split(buf, counts):
    out, o = [], 0
    for c in counts:
        out.append(buf[o:o + c])
        o += c
    return out


def exchange_dist(send: np.ndarray, send_counts, recv_counts, group=None) -> np.ndarray:
    """One message per rank pair through torch.distributed (gloo on host tensors; NCCL on the
    current CUDA device)."""
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    src = torch.from_numpy(np.ascontiguousarray(send, np.float32)).to(dev)
    dst = torch.empty(int(sum(recv_counts)), dtype=torch.float32, device=dev)
    dist.all_to_all_single(dst, src, output_split_sizes=list(recv_counts),
                           input_split_sizes=list(send_counts), group=group)
    return dst.cpu().numpy()


def check_sea_status(case) -> None:
    """W3SCAT skips a sea point with MAPSTA = 0, so its owner would receive a stale send-back
    value under W3_MPI; WW3 never numbers such a cell as a sea point, and the fork's XYP3_MPI
    stops on one (the reference's PATCH.md:2480-2487). So does this."""
    nsea = case["nsea"]
    ixy = np.asarray(case["mapsf"])[2 * nsea:3 * nsea]
    if np.any(np.asarray(case["mapsta"])[ixy - 1] == 0):
        raise ValueError("a sea point has MAPSTA = 0: W3XYP3 under W3_MPI stops there")


def step_dist(L, igrid, case, va, iappro, group=None) -> int:
    """Steps 1-5 on this process's rank of ``group``; va is this rank's VA(NSPEC, 0:NSEALM),
    bound as the resident VA of grid igrid. Returns the status of ww_xyp3_batch_mpi (every rank
    takes part in both exchanges whatever it is)."""
    import torch.distributed as dist

    check_sea_status(case)
    naproc, iaproc = dist.get_world_size(group), dist.get_rank(group) + 1
    lay = layout(iappro, naproc, iaproc, case["nsea"])
    sent = pack(L, igrid, va, lay)
    rbuf = exchange_dist(sent, lay.send_counts, lay.recv_counts, group)
    rc, sbuf = propagate(L, igrid, case, va, lay, rbuf)
    back = exchange_dist(sbuf if rc == 0 else np.zeros(lay.nbuf, np.float32),
                         lay.recv_counts, lay.send_counts, group)
    if rc == 0:
        unpack(L, igrid, va, lay, back)
    return rc


def step_local(L, igrids, case, vas, iappro) -> list:
    """Steps 1-5 for all NAPROC ranks emulated in one process, one after another (rank IP's
    resident VA is grid igrids[IP-1], bound to vas[IP-1]). Returns each rank's status."""
    check_sea_status(case)
    naproc = len(vas)
    lays = [layout(iappro, naproc, ip, case["nsea"]) for ip in range(1, naproc + 1)]
    sent = [_split(pack(L, igrids[i], vas[i], lays[i]), lays[i].send_counts)
            for i in range(naproc)]
    # Rank IP receives, in rank order, what each other rank sent to it.
    rbufs = [np.concatenate([sent[j][i] for j in range(naproc) if j != i] or
                            [np.zeros(0, np.float32)]) for i in range(naproc)]
    rcs, back = [], []
    for i in range(naproc):
        rc, sbuf = propagate(L, igrids[i], case, vas[i], lays[i], rbufs[i])
        rcs.append(rc)
        back.append(_split(sbuf, lays[i].recv_counts))
    for i in range(naproc):
        buf = np.concatenate([back[j][i] for j in range(naproc) if j != i] or
                             [np.zeros(0, np.float32)])
        unpack(L, igrids[i], vas[i], lays[i], buf)
    return rcs
