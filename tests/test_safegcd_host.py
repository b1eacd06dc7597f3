"""Host build of the divstep inversion (impeller_b200/csrc/safegcd.cuh).

The header is written for host and device alike; here g++ compiles it for
the CPU and its inverses are checked against Python's big-integer pow(x, -1,
p) on every field the library inverts in (BN254 Fq and Fr, BLS12-381 Fq and
Fr): edge values (1, 2, p - 1, p - 2, powers of two, values with long runs of
zero or one bits) and seeded random values.  The device copy of the same code
is checked on the GPU through the field test hook (tests/test_gpu_parity.py).
"""
import ctypes
import os
import random
import shutil
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(HERE, "..", "impeller_b200", "csrc", "safegcd.cuh")

SHIM = r"""
#include "safegcd.cuh"
extern "C" void sg_inv8(const uint32_t *x, const uint32_t *p, uint32_t *out) { ec::sg::inverse<8>(x, p, out); }
extern "C" void sg_inv12(const uint32_t *x, const uint32_t *p, uint32_t *out) { ec::sg::inverse<12>(x, p, out); }
"""

FIELDS = {
    "bn254_fq": (0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47, 8),
    "bn254_fr": (0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001, 8),
    "bls12381_fr": (0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001, 8),
    "bls12381_fq": (0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F624_1EABFFFEB153FFFFB9FEFFFFFFFFAAAB, 12),
}


@pytest.fixture(scope="module")
def lib():
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tempfile.mkdtemp(prefix="sg_")
    src = os.path.join(d, "shim.cpp")
    with open(src, "w") as f:
        f.write(SHIM)
    so = os.path.join(d, "libsg.so")
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I", os.path.dirname(HEADER), src, "-o", so],
                   check=True)
    return ctypes.CDLL(so)


def words(x: int, n: int):
    return (ctypes.c_uint32 * n)(*[(x >> (32 * i)) & 0xFFFFFFFF for i in range(n)])


def value(w) -> int:
    return sum(int(v) << (32 * i) for i, v in enumerate(w))


def inv(lib, x: int, p: int, n: int) -> int:
    out = (ctypes.c_uint32 * n)()
    fn = lib.sg_inv8 if n == 8 else lib.sg_inv12
    fn(words(x, n), words(p, n), out)
    return value(out)


def cases(p: int, seed: int):
    bits = p.bit_length()
    edge = [1, 2, 3, p - 1, p - 2, (p - 1) // 2, (p + 1) // 2]
    edge += [1 << k for k in range(0, bits - 1, 7)]
    edge += [(1 << k) - 1 for k in range(2, bits - 1, 11)]
    edge += [p - (1 << k) for k in range(0, bits - 2, 13)]
    rng = random.Random(seed)
    edge += [rng.randrange(1, p) for _ in range(400)]
    # small values and values just below p (long common runs with p)
    edge += [rng.randrange(1, 1 << 40) for _ in range(50)] + [p - rng.randrange(1, 1 << 40) for _ in range(50)]
    return edge


@pytest.mark.parametrize("field", sorted(FIELDS))
def test_inverse_matches_bigint(lib, field):
    p, n = FIELDS[field]
    for k, x in enumerate(cases(p, seed=sum(field.encode()))):
        got = inv(lib, x, p, n)
        assert got == pow(x, -1, p), f"{field} case {k}: x={x:#x}"
        assert got < p


@pytest.mark.parametrize("field", sorted(FIELDS))
def test_inverse_of_zero_is_zero(lib, field):
    p, n = FIELDS[field]
    assert inv(lib, 0, p, n) == 0
