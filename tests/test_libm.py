"""The device expf (ww3-gpu_b200/csrc/libm_dev.cuh) against this host's glibc expf.

W3SNL1's CONS calls expf (reference snl1_team.hpp:386-390); on the CPU that is glibc. The header
compiles for host and device from one source (fma() on the host, __fma_rn on the device), so
comparing its host build with glibc checks the bits the kernel computes. The full 2^32 sweep
takes about half a minute on 8 cores; the default run checks every 61st bit pattern
(~70 M inputs, every region of the float line), WWB_LIBM_FULL=1 checks all.
"""

import os
import re
import pathlib
import struct
import subprocess
from decimal import Decimal, getcontext

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
HDR = ROOT / "ww3-gpu_b200" / "csrc" / "libm_dev.cuh"


def test_exp2f_table_is_2_pow_i_over_32():
    """Each entry is 2^(i/32) rounded to nearest double, with i << 47 subtracted from its bits."""
    getcontext().prec = 60
    ln2 = Decimal(2).ln()
    text = HDR.read_text()
    start = text.index("#define WWB_EXP2F_TAB")
    body = text[start:text.index("}", start)]
    entries = [int(m, 16) for m in re.findall(r"0x([0-9a-f]{16})ULL", body)]
    assert len(entries) == 32
    for i, got in enumerate(entries):
        v = float((ln2 * i / 32).exp())
        u = struct.unpack("<Q", struct.pack("<d", v))[0]
        assert got == (u - (i << 47)) & 0xFFFFFFFFFFFFFFFF, i


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = tmp_path_factory.mktemp("libm") / "libm_check"
    subprocess.run(["/usr/bin/g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-math-errno",
                    "-fopenmp", str(ROOT / "tests" / "libm_check.cpp"), "-o", str(exe)],
                   check=True)
    return exe


def test_expf_equals_glibc(checker):
    stride = "1" if os.environ.get("WWB_LIBM_FULL") == "1" else "61"
    out = subprocess.run([str(checker), stride], check=True, capture_output=True, text=True).stdout
    default = int(re.search(r"default (\d+)", out).group(1))
    lines = [ln for ln in out.splitlines() if ln.startswith("variant")]
    per_variant = {int(ln.split()[1]): int(ln.split()[2]) for ln in lines}
    assert per_variant[default] == 0, out
