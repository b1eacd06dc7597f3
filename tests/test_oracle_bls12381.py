"""The CPU oracle on the reference's second curve, BLS12-381 G1, pinned.

The reference carries BLS12-381 parameters (core/src/common/mont/src/
bls12381_fq.cuh, bls12381_fr.cuh; core/src/common/curve/src/bls12381.cuh) and
lists the curve among its MSM library targets (core/src/msm/xmake.lua) and in
its operator (core/src/msm.rs:24-34), but ships no BLS12-381 known-answer
vectors.  The pins are therefore:
  1. the published curve constants (generator on the curve, r * G = O);
  2. MSM outputs computed with the reference's own host arithmetic
     (tests/golden/msm_golden_bls12381.json, written by make_golden.py);
  3. pure-Python big integers on small inputs;
  4. when the reference sources are mounted, the reference's field and point
     arithmetic on fresh random inputs (oracle/_ref/libref_bn254.so).
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
C = O.BLS12381
R384 = 1 << 384

GX = 0x17f1d3a73197d7942695638c4fa9ac0fc3688c4f9774b905a14e3a3f171bac586c55e83ff97a1aeffb3af00adb22c6bb
GY = 0x08b3f481e3aaa0f1a09e30ed741d8ae4fcf5e095d5d00af600db18cb2c04b3edd03cc744a2888ae40caa232946c5e7e1


def rows(hexrows, width):
    return np.array([[int(r[8 * i:8 * i + 8], 16) for i in range(width)] for r in hexrows],
                    dtype=np.uint32).reshape(-1, width)


def fq_arr(xs):
    return O.ints_to_array([x * R384 % O.P_BLS for x in xs], 12)


def fq_ints(a):
    ri = pow(R384, -1, O.P_BLS)
    return [O.limbs_to_int(r) * ri % O.P_BLS for r in np.asarray(a).reshape(-1, 12)]


def test_curve_constants():
    p, r = O.P_BLS, O.R_BLS
    assert p.bit_length() == 381 and r.bit_length() == 255
    assert (GY * GY - GX ** 3 - 4) % p == 0
    assert O.py_mul(r, (GX, GY), p) is None
    g = O.py_point_to_limbs((GX, GY), C)
    assert O.point_op(O.PT_ONCURVE, g, curve=C)[0, 0] == 1
    # r * G = identity through the oracle's own scalar multiplication
    assert not O.point_op(O.PT_SMUL, g, O.int_to_limbs(r)[None], curve=C).any()


def test_fq_ops_vs_python_ints():
    rng = np.random.default_rng(11)
    p = O.P_BLS
    xs = [int.from_bytes(rng.bytes(48), "little") % p for _ in range(64)] + [0, 1, p - 1]
    ys = [int.from_bytes(rng.bytes(48), "little") % p for _ in range(64)] + [p - 1, 0, p - 1]
    a, b = fq_arr(xs), fq_arr(ys)
    assert fq_ints(O.field_op(O.BLS_FQ, O.ADD, a, b)) == [(x + y) % p for x, y in zip(xs, ys)]
    assert fq_ints(O.field_op(O.BLS_FQ, O.SUB, a, b)) == [(x - y) % p for x, y in zip(xs, ys)]
    assert fq_ints(O.field_op(O.BLS_FQ, O.MUL, a, b)) == [x * y % p for x, y in zip(xs, ys)]
    assert fq_ints(O.field_op(O.BLS_FQ, O.SQR, a)) == [x * x % p for x in xs]
    assert fq_ints(O.field_op(O.BLS_FQ, O.NEG, a)) == [-x % p for x in xs]
    inv = fq_ints(O.field_op(O.BLS_FQ, O.INV, a))
    assert all(x == 0 or x * v % p == 1 for x, v in zip(xs, inv))
    plain = O.ints_to_array(xs, 12)
    assert (O.field_op(O.BLS_FQ, O.TO_MONT, plain) == a).all()
    assert (O.field_op(O.BLS_FQ, O.FROM_MONT, a) == plain).all()


def test_fr_ops_vs_python_ints():
    rng = np.random.default_rng(12)
    r = O.R_BLS
    xs = [int.from_bytes(rng.bytes(32), "little") % r for _ in range(64)] + [0, 1, r - 1]
    ys = [int.from_bytes(rng.bytes(32), "little") % r for _ in range(64)] + [r - 1, r - 1, r - 1]
    a = O.ints_to_array([O.to_mont(x, r) for x in xs])
    b = O.ints_to_array([O.to_mont(y, r) for y in ys])

    def ints(arr):
        return [O.from_mont(O.limbs_to_int(v), r) for v in arr]

    assert ints(O.field_op(O.BLS_FR, O.ADD, a, b)) == [(x + y) % r for x, y in zip(xs, ys)]
    assert ints(O.field_op(O.BLS_FR, O.SUB, a, b)) == [(x - y) % r for x, y in zip(xs, ys)]
    assert ints(O.field_op(O.BLS_FR, O.MUL, a, b)) == [x * y % r for x, y in zip(xs, ys)]
    assert ints(O.field_op(O.BLS_FR, O.NEG, a)) == [-x % r for x in xs]


def test_generators_are_r_times_g_and_pinned():
    rr = O.gen_scalars(3, seed=0, stream=0, mont=False, curve=C)
    pts = O.gen_points(3, seed=0, curve=C)
    for i in range(3):
        want = O.py_point_to_limbs(O.py_mul(O.limbs_to_int(rr[i]), (GX, GY), O.P_BLS), C)
        assert (pts[i] == want).all()
    assert all(O.limbs_to_int(v) < O.R_BLS for v in O.gen_scalars(256, seed=4, stream=1, mont=False, curve=C))
    g = json.load(open(os.path.join(GOLD, "generators_bls12381.json")))
    assert (O.gen_points(4, seed=0, curve=C) == rows(g["srs_points_seed0_first4"], 24)).all()
    assert (O.gen_scalars(4, seed=0, stream=0, mont=False, curve=C) == rows(g["srs_r_seed0_first4"], 8)).all()
    assert (O.gen_scalars(4, seed=0, stream=1, curve=C) == rows(g["uniform_seed0_stream1_first4_mont"], 8)).all()
    sk = O.gen_scalars(32, seed=0, stream=2, dist=O.DIST_SKEWED, mont=False, curve=C)
    assert (sk == rows(g["skewed_seed0_stream2_first32_canonical"], 8)).all()


def test_golden_msm_cases():
    gold = json.load(open(os.path.join(GOLD, "msm_golden_bls12381.json")))
    assert len(gold["cases"]) >= 10
    for case in gold["cases"]:
        pts = rows(case["points"], 24)
        sc = rows(case["scalars"], 8)
        want = rows([case["result"]], 24)[0]
        assert (O.msm(pts, sc, threads=3, curve=C) == want).all(), case["name"]
        assert (O.msm_naive(pts, sc, curve=C) == want).all(), case["name"]


def test_msm_vs_python_ints():
    pts = O.gen_points(12, seed=3, curve=C)
    sc = O.gen_scalars(12, seed=3, stream=9, curve=C)
    assert (O.msm(pts, sc, curve=C) == O.py_msm(pts, sc, curve=C)).all()


@pytest.mark.parametrize("n", [1, 3, 4, 33, 300, 2049])
def test_best_multiexp_thread_split(n):
    pts = O.gen_points(n, seed=1, curve=C)
    sc = O.gen_scalars(n, seed=1, stream=2, curve=C)
    a = O.msm(pts, sc, threads=1, curve=C)
    assert (a == O.msm(pts, sc, threads=5, curve=C)).all()
    if n <= 64:
        assert (a == O.msm_naive(pts, sc, curve=C)).all()


def test_precompute_tables():
    pts = O.gen_points(4, seed=2, curve=C)
    tabs = O.precompute(pts, shift=9, n_tables=3, curve=C)
    assert (tabs[0] == pts).all()
    for j in (1, 2):
        k = O.int_to_limbs(1 << (9 * j))
        assert (tabs[j] == O.point_op(O.PT_SMUL, pts, np.repeat(k[None], 4, 0), curve=C)).all()


@pytest.mark.skipif(not O.ref_available(), reason="reference sources not mounted")
def test_oracle_vs_reference_arithmetic_random():
    rng = np.random.default_rng(8)
    p, r = O.P_BLS, O.R_BLS
    xs = [int.from_bytes(rng.bytes(48), "little") % p for _ in range(100)]
    ys = [int.from_bytes(rng.bytes(48), "little") % p for _ in range(100)]
    a, b = fq_arr(xs), fq_arr(ys)
    for op in (O.ADD, O.SUB, O.MUL, O.SQR, O.NEG, O.TO_MONT, O.FROM_MONT, O.INV):
        assert (O.field_op(O.BLS_FQ, op, a, b) == O.field_op(O.BLS_FQ, op, a, b, use_ref=True)).all(), op
    xs = [int.from_bytes(rng.bytes(32), "little") % r for _ in range(100)]
    ys = [int.from_bytes(rng.bytes(32), "little") % r for _ in range(100)]
    a, b = O.ints_to_array(xs), O.ints_to_array(ys)
    for op in (O.ADD, O.SUB, O.MUL, O.SQR, O.NEG, O.TO_MONT, O.FROM_MONT, O.INV):
        assert (O.field_op(O.BLS_FR, op, a, b) == O.field_op(O.BLS_FR, op, a, b, use_ref=True)).all(), op
    pts = O.gen_points(64, seed=6, curve=C)
    q = O.gen_points(64, seed=7, curve=C)
    q[::9] = pts[::9]  # P + P takes the doubling branch
    assert (O.point_op(O.PT_ADD, pts, q, curve=C) == O.ref_point_op(O.PT_ADD, pts, q, curve=C)).all()
    assert (O.point_op(O.PT_DBL, pts, curve=C) == O.ref_point_op(O.PT_DBL, pts, curve=C)).all()
    sc = O.gen_scalars(32, seed=6, stream=5, curve=C)
    assert (O.msm(pts[:32], sc, curve=C) == O.ref_msm_naive(pts[:32], sc, curve=C)).all()
