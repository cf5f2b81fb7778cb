"""Convert the reference's frozen W3SNL1 golden vector into tests/golden/snl1_nk25_nth24.npz.

The source is ww3-gpu's kokkos/tests/fixtures/snl1_nk25_nth24.bin: a WAVEWATCH III sea state
(NK=25, NTH=24, three points at 1000, 50 and 10 m depth) together with the Fortran INSNL1
tables and the Fortran W3SNL1 answers S and D for it. Its layout is documented in
kokkos/tests/fixtures/README.md (section "Binary layout"): little-endian int32/float32, no
record markers, index tables 1-based as Fortran holds them. This script is the only place
that reads that layout; it stores the index tables 0-based (Fortran value minus one), the
convention of kokkos/src/ww_kokkos/snl1_tables.hpp:5-12 and of this project's C ABI.

Run it where the reference is mounted:
    python tests/golden/make_golden.py /path/to/ww3-gpu
The .npz it writes is committed, so the tests never read the reference at run time.
"""

import os
import pathlib
import sys

import numpy as np

IPIM_NAMES = ["ip11", "ip12", "ip13", "ip14", "im11", "im12", "im13", "im14",
              "ip21", "ip22", "ip23", "ip24", "im21", "im22", "im23", "im24"]
IC_NAMES = ["ic11", "ic21", "ic31", "ic41", "ic51", "ic61", "ic71", "ic81",
            "ic12", "ic22", "ic32", "ic42", "ic52", "ic62", "ic72", "ic82"]


def read_bin(path):
    b = pathlib.Path(path).read_bytes()
    off = 0

    def take(dtype, n):
        nonlocal off
        a = np.frombuffer(b, dtype=dtype, count=n, offset=off).copy()
        off += a.nbytes
        return a

    magic, nk, nth, npts = take("<i4", 4)
    if magic != 0x534E4C31:
        raise ValueError("not an SNL1 fixture")
    nspec = nk * nth
    out = {"nk": nk, "nth": nth, "npts": npts}
    hdr = take("<f4", 10)
    for name, v in zip(["xfr", "dth", "lam", "snlc1", "kdcon", "kdmn", "snls1", "snls2",
                        "snls3", "fachfe"], hdr):
        out[name] = np.float32(v)
    out["sig"] = take("<f4", nk)
    scal = take("<i4", 5)
    out["scal"] = scal  # nfr, nfrhgh, nfrchg, nspecx, nspecy
    nspecx = int(scal[3])
    out["wts"] = take("<f4", 19)  # dal1..3, awg(8), swg(8)
    out["ipim"] = take("<i4", 16 * nspecx).reshape(16, nspecx) - 1
    out["ic"] = take("<i4", 16 * nspec).reshape(16, nspec) - 1
    out["af11"] = take("<f4", nspecx)
    kd, cg, a, s, d = [], [], [], [], []
    for _ in range(npts):
        kd.append(take("<f4", 1)[0])
        cg.append(take("<f4", nk))
        a.append(take("<f4", nspec))
        s.append(take("<f4", nspec))
        d.append(take("<f4", nspec))
    if off != len(b):
        raise ValueError(f"trailing bytes: read {off} of {len(b)}")
    # Column-major (nspec, npts) in memory = row-major (npts, nspec) here.
    out["kdmean"] = np.array(kd, dtype=np.float32)
    out["cg"] = np.stack(cg).astype(np.float32)
    out["a"] = np.stack(a).astype(np.float32)
    out["s"] = np.stack(s).astype(np.float32)
    out["d"] = np.stack(d).astype(np.float32)
    return out


def main():
    if len(sys.argv) > 1:
        root = pathlib.Path(sys.argv[1])
    elif os.environ.get("WW_REFERENCE_ROOT"):
        root = pathlib.Path(os.environ["WW_REFERENCE_ROOT"])
    else:
        root = pathlib.Path(__file__).resolve().parents[3] / "reference"
    src = root / "kokkos/tests/fixtures/snl1_nk25_nth24.bin"
    dst = pathlib.Path(__file__).with_name("snl1_nk25_nth24.npz")
    g = read_bin(src)
    np.savez_compressed(dst, **{k: np.asarray(v) for k, v in g.items()})
    print(f"wrote {dst} ({dst.stat().st_size} bytes) from {src}")


if __name__ == "__main__":
    main()
