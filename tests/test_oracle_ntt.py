"""The CPU oracle for the NTT operator, pinned before it is trusted.

Pins: the definition of the transform (a naive O(n^2) DFT over Python
integers), the reference's own host code for the recompute tables
(gen_pq_omegas of core/src/ntt/src/precompute.cuh, run from the reference's
library built here, oracle/_ref/libref_ntt_bn254_fr.so, when present), and
the algebraic identities an NTT must satisfy (inverse round trip, linearity,
convolution theorem).  GPU parity with the reference's own ssip_ntt kernel is
in tests/test_gpu_ntt.py."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

REF_NTT = os.path.join(os.path.dirname(O.__file__), "_ref", "libref_ntt_bn254_fr.so")
MONT = 1 << 256


def to_ints(a, m):
    ri = pow(MONT, -1, m)
    return [O.limbs_to_int(r) * ri % m for r in np.asarray(a).reshape(-1, 8)]


def from_ints(xs, m):
    return O.ints_to_array([x * MONT % m for x in xs])


def naive_dft(xs, w, m):
    n = len(xs)
    return [sum(xs[j] * pow(w, j * k, m) for j in range(n)) % m for k in range(n)]


@pytest.mark.parametrize("field", [O.FR, O.BLS_FR])
@pytest.mark.parametrize("log_n", [0, 1, 2, 3, 4, 6, 7])
def test_ntt_matches_definition(field, log_n):
    m = O.NTT_FIELDS[field][2]
    rng = np.random.default_rng(log_n + 10 * field)
    xs = [int.from_bytes(rng.bytes(32), "little") % m for _ in range(1 << log_n)]
    w = O.root_of_unity(log_n, field)
    got = O.ntt(from_ints(xs, m), O.mont_limbs(w, field), field)
    assert to_ints(got, m) == naive_dft(xs, w, m)


def test_bn254_fq_two_point():
    # BN254 Fq has 2-adicity 1: only the 2-point transform exists
    m = O.P
    w = O.root_of_unity(1, O.FQ)
    assert w == m - 1
    got = O.ntt(from_ints([5, 7], m), O.mont_limbs(w, O.FQ), O.FQ)
    assert to_ints(got, m) == [12, (5 - 7) % m]


def test_inverse_roundtrip_and_linearity():
    m = O.R_MOD
    log_n = 10
    n = 1 << log_n
    rng = np.random.default_rng(3)
    xs = [int.from_bytes(rng.bytes(32), "little") % m for _ in range(n)]
    ys = [int.from_bytes(rng.bytes(32), "little") % m for _ in range(n)]
    w = O.root_of_unity(log_n)
    fx = O.ntt(from_ints(xs, m), O.mont_limbs(w))
    back = to_ints(O.ntt(fx, O.mont_limbs(pow(w, -1, m))), m)
    ninv = pow(n, -1, m)
    assert [v * ninv % m for v in back] == xs
    fy = O.ntt(from_ints(ys, m), O.mont_limbs(w))
    fs = O.ntt(from_ints([(a + 3 * b) % m for a, b in zip(xs, ys)], m), O.mont_limbs(w))
    assert to_ints(fs, m) == [(a + 3 * b) % m for a, b in zip(to_ints(fx, m), to_ints(fy, m))]


def test_convolution_theorem():
    m = O.R_MOD
    n = 64
    rng = np.random.default_rng(4)
    a = [int(v) for v in rng.integers(0, 1000, n // 2)] + [0] * (n // 2)
    b = [int(v) for v in rng.integers(0, 1000, n // 2)] + [0] * (n // 2)
    w = O.root_of_unity(6)
    fa = to_ints(O.ntt(from_ints(a, m), O.mont_limbs(w)), m)
    fb = to_ints(O.ntt(from_ints(b, m), O.mont_limbs(w)), m)
    prod = O.ntt(from_ints([x * y % m for x, y in zip(fa, fb)], m), O.mont_limbs(pow(w, -1, m)))
    conv = [v * pow(n, -1, m) % m for v in to_ints(prod, m)]
    want = [sum(a[i] * b[k - i] for i in range(k + 1)) for k in range(n)]
    assert conv == want


def test_roots_pq_omegas_distribute():
    m = O.R_MOD
    w = O.root_of_unity(12)
    roots = to_ints(O.ntt_roots(100, O.mont_limbs(w)), m)
    assert roots == [pow(w, i, m) for i in range(100)]
    pq, om = O.pq_omegas(5, 1 << 12, O.mont_limbs(w))
    assert to_ints(pq, m) == [pow(w, i << 7, m) for i in range(16)]
    assert to_ints(om, m) == [pow(w, 1 << i, m) for i in range(32)]
    xs = list(range(1, 11))
    pw = [3, 5, 7]
    got = to_ints(O.distribute_powers(from_ints(xs, m), from_ints(pw, m), begin=4, poly_len=12), m)
    assert got == [xs[i] * pw[((4 + i) % 12) % 3] % m for i in range(10)]


REF_NTT_BLS = os.path.join(os.path.dirname(O.__file__), "_ref", "libref_ntt_bls12381_fr.so")


@pytest.mark.parametrize("field,path", [(O.FR, REF_NTT), (O.BLS_FR, REF_NTT_BLS)])
def test_pq_omegas_match_reference_host_code(field, path):
    """gen_pq_omegas is host code in the reference (precompute.cuh:100-125):
    run it from the reference's own library, no GPU involved."""
    if not os.path.exists(path):
        pytest.skip("reference NTT library not built")
    ref = ctypes.CDLL(path)
    ref.gen_pq_omegas.restype = None
    ref.gen_pq_omegas.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p]
    for log_n, deg in ((12, 5), (20, 9), (3, 1), (24, 10)):
        w = O.mont_limbs(O.root_of_unity(log_n, field), field)
        pq = np.zeros(((1 << deg) >> 1 or 1, 8), np.uint32)
        om = np.zeros((32, 8), np.uint32)
        u = np.ascontiguousarray(w, dtype=np.uint32)
        ref.gen_pq_omegas(pq.ctypes.data, om.ctypes.data, deg, 1 << log_n, u.ctypes.data)
        want_pq, want_om = O.pq_omegas(deg, 1 << log_n, w, field)
        assert (om == want_om).all(), (log_n, deg)
        assert (pq[: want_pq.shape[0]] == want_pq).all(), (log_n, deg)
