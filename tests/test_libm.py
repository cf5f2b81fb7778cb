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


def _mismatches(checker, fn, stride):
    out = subprocess.run([str(checker), fn, str(stride)], check=True, capture_output=True,
                         text=True).stdout
    default = int(re.search(r"default (\d+)", out).group(1))
    lines = [ln for ln in out.splitlines() if ln.startswith("variant")]
    per_variant = {int(ln.split()[1]): int(ln.split()[2]) for ln in lines}
    return per_variant, default, out


FULL = os.environ.get("WWB_LIBM_FULL") == "1"


def test_expf_equals_glibc(checker):
    per_variant, default, out = _mismatches(checker, "expf", 1 if FULL else 61)
    assert per_variant[default] == 0, out


@pytest.mark.parametrize("fn", ["logf", "sincosf", "tanhf", "atanf", "log10f", "sinhf", "coshf"])
def test_unary_equals_glibc(checker, fn):
    """Every 61st bit pattern (all 2^32 with WWB_LIBM_FULL=1); sincosf also against a lone
    sinf and cosf, which the reference calls as separate functions."""
    per_variant, _, out = _mismatches(checker, fn, 1 if FULL else 61)
    assert per_variant[0] == 0 and per_variant[1] == 0, out


@pytest.mark.parametrize("fn", ["powf", "atan2f"])
def test_binary_equals_glibc(checker, fn):
    """Seeded argument pairs: 2^32/64 of them (2^32/4 with WWB_LIBM_FULL=1)."""
    per_variant, _, out = _mismatches(checker, fn, 4 if FULL else 64)
    assert per_variant[0] == 0, out


def _decimal_table(name):
    text = HDR.read_text()
    start = text.index(f"#define {name}")
    body = text[start:text.index("}", start)]
    return [float.fromhex(m) for m in re.findall(r"(-?0x[0-9a-f.]+p[+-]?\d+)", body)]


def test_log_tables_are_generated_from_invc():
    """ln(c) and log2(c) of the logf / powf subintervals are -ln(invc) and -log2(invc) of the
    published 1/c values, rounded to double."""
    getcontext().prec = 60
    invc = _decimal_table("WWB_LOG_INVC")
    logc = _decimal_table("WWB_LOG_LOGC")
    log2c = _decimal_table("WWB_LOG2_LOGC")
    assert len(invc) == len(logc) == len(log2c) == 16
    ln2 = Decimal(2).ln()
    for i in range(16):
        lnc = -Decimal(invc[i]).ln()
        assert float(lnc) == logc[i], i
        assert float(lnc / ln2) == log2c[i], i


def test_inv_pio4_is_two_over_pi():
    """The sincosf reduction table is 2/pi's binary fraction in 32-bit windows 8 bits apart."""
    getcontext().prec = 100
    text = HDR.read_text()
    start = text.index("#define WWB_INV_PIO4")
    body = text[start:text.index("}", start)]
    words = [int(m, 16) for m in re.findall(r"0x([0-9a-f]+)u", body)]
    # pi by Machin's formula
    def arctan_inv(n):
        x = Decimal(1) / n
        s, t, k = x, x, 1
        while True:
            t *= -x * x
            k += 2
            d = t / k
            if abs(d) < Decimal(10) ** -95:
                return s
            s += d
    pi = 16 * arctan_inv(5) - 4 * arctan_inv(239)
    f, b = 2 / pi, []
    for _ in range(30):
        f *= 256
        b.append(int(f))
        f -= int(f)
    for j, w in enumerate(words):
        want = 0
        for q in range(4):
            idx = j - 3 + q
            want = (want << 8) | (b[idx] if idx >= 0 else 0)
        assert w == want, j


def test_exp2_64_table():
    """2^(j/64) of the double exp as double-double: hi rounded to double, lo the remainder."""
    getcontext().prec = 60
    vals = _decimal_table("WWB_EXP2_64_TAB")
    assert len(vals) == 128
    for j in range(64):
        v = Decimal(2) ** (Decimal(j) / 64)
        hi = float(v)
        assert vals[2 * j] == hi, j
        assert vals[2 * j + 1] == float(v - Decimal(hi)), j
