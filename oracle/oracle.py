"""Python access to the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker.  The CUDA product
path never routes through it.

``liboracle.so`` (``bn254_oracle.c``) restates the reference's CPU MSM,
``core/tests/msm_halo2.rs:63-208`` (halo2 ``multiexp_serial`` /
``best_multiexp``), plus the seeded synthetic-input generators.
``_ref/libref_bn254.so`` (built only where the reference sources exist) wraps
the reference's own host field/curve arithmetic
(``core/src/common/mont/src/field.cuh``,
``core/src/common/curve/src/curve_xyzz.cuh``) to pin the restatement.

All arrays use the C ABI layout of ``core/src/msm/src/msm.h``: field elements
are 8 little-endian uint32 limbs in Montgomery form (R = 2^256), affine points
are 16 uint32 (x then y), the identity point is all zeros.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_bn254.so")

P = 21888242871839275222246405745257275088696311157297823662689037894645226208583
R_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617
MONT_R = 1 << 256

# BLS12-381 (the reference's second curve): p (381 bits, 12 u32 limbs,
# R = 2^384) and the group order r (255 bits, 8 limbs, R = 2^256).
P_BLS = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab
R_BLS = 0x73eda753299d7d483339d80809a1d80553bda402fffe5bfeffffffff00000001

BN254, BLS12381 = 0, 1
# per curve: symbol prefix, base modulus, scalar modulus, Fq words, Montgomery R of Fq
CURVES = {BN254: ("orc_", P, R_MOD, 8, 1 << 256), BLS12381: ("orc_bls_", P_BLS, R_BLS, 12, 1 << 384)}

# fields: BN254 Fq, Fr; BLS12-381 Fq, Fr
FQ, FR, BLS_FQ, BLS_FR = 0, 1, 2, 3
ADD, SUB, MUL, SQR, NEG, TO_MONT, FROM_MONT, INV, POW = range(9)
PT_ADD, PT_DBL, PT_NEG, PT_SMUL, PT_ONCURVE = range(5)

DIST_UNIFORM, DIST_SKEWED = 0, 1
SRS_STREAM = 0

_u32p = ctypes.POINTER(ctypes.c_uint32)
_lib = None
_ref = None


def build() -> None:
    """Compile liboracle.so (and the reference harness when possible)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = ctypes.CDLL(ORACLE_SO)
        for pre in ("orc_", "orc_bls_"):
            getattr(L, pre + "ntt").argtypes = [ctypes.c_int, _u32p, ctypes.c_uint32, _u32p]
            getattr(L, pre + "ntt_roots").argtypes = [ctypes.c_int, _u32p, ctypes.c_uint64, _u32p]
            getattr(L, pre + "pq_omegas").argtypes = [ctypes.c_int, _u32p, _u32p, ctypes.c_uint32, ctypes.c_uint64,
                                                      _u32p]
            getattr(L, pre + "field_op").argtypes = [ctypes.c_int, ctypes.c_int, _u32p, _u32p, _u32p,
                                                     ctypes.c_uint64]
            getattr(L, pre + "point_op").argtypes = [ctypes.c_int, _u32p, _u32p, _u32p, ctypes.c_uint64]
            getattr(L, pre + "gen_scalars").argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                                        ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _u32p,
                                                        ctypes.c_int]
            getattr(L, pre + "gen_points").argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, _u32p,
                                                       ctypes.c_int]
            getattr(L, pre + "msm_halo2").argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p, ctypes.c_int]
            getattr(L, pre + "msm_naive").argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p]
            getattr(L, pre + "precompute").argtypes = [_u32p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                                       _u32p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    """The reference-arithmetic harness; None when it was not built here."""
    global _ref
    if _ref is None and ref_available():
        L = ctypes.CDLL(REF_SO)
        L.ref_field_op.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, _u32p, _u32p, ctypes.c_uint64]
        L.ref_point_add.argtypes = [_u32p, _u32p, _u32p, ctypes.c_uint64]
        L.ref_point_dbl.argtypes = [_u32p, _u32p, ctypes.c_uint64]
        L.ref_msm_naive.argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p]
        L.ref_bls_point_add.argtypes = [_u32p, _u32p, _u32p, ctypes.c_uint64]
        L.ref_bls_point_dbl.argtypes = [_u32p, _u32p, ctypes.c_uint64]
        L.ref_bls_msm_naive.argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p]
        _ref = L
    return _ref


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_u32p)


def default_threads() -> int:
    return os.cpu_count() or 1


# ---------------------------------------------------------------- conversions

def int_to_limbs(x: int, words: int = 8) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(words)], dtype=np.uint32)


def limbs_to_int(a) -> int:
    a = np.asarray(a, dtype=np.uint32).reshape(-1)
    return sum(int(v) << (32 * i) for i, v in enumerate(a))


def ints_to_array(xs, words: int = 8) -> np.ndarray:
    return np.stack([int_to_limbs(x, words) for x in xs]).astype(np.uint32) if len(xs) else \
        np.zeros((0, words), dtype=np.uint32)


def to_mont(x: int, m: int) -> int:
    return x * MONT_R % m


def from_mont(x: int, m: int) -> int:
    return x * pow(MONT_R, -1, m) % m


# ------------------------------------------------------------------- wrappers

def _fn(curve: int, name: str):
    return getattr(lib(), CURVES[curve][0] + name)


def _pw(curve: int) -> int:
    """u32 words per affine point."""
    return 2 * CURVES[curve][3]


def field_op(field: int, op: int, a: np.ndarray, b: np.ndarray | None = None, use_ref: bool = False) -> np.ndarray:
    """Element-wise field operation; field FQ / FR (BN254) or BLS_FQ / BLS_FR."""
    words = 12 if field == BLS_FQ else 8
    a = np.ascontiguousarray(a, dtype=np.uint32).reshape(-1, words)
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.uint32).reshape(-1, words)
    out = np.zeros_like(a)
    if use_ref:
        fn, f = ref_lib().ref_field_op, field
    elif field in (BLS_FQ, BLS_FR):
        fn, f = _fn(BLS12381, "field_op"), field - BLS_FQ
    else:
        fn, f = _fn(BN254, "field_op"), field
    rc = fn(f, op, _ptr(a), _ptr(bb), _ptr(out), a.shape[0])
    if rc != 0:
        raise RuntimeError(f"field_op rc={rc}")
    return out


def point_op(op: int, p: np.ndarray, q: np.ndarray | None = None, curve: int = BN254) -> np.ndarray:
    pw = _pw(curve)
    p = np.ascontiguousarray(p, dtype=np.uint32).reshape(-1, pw)
    qq = None
    if q is not None:
        qq = np.ascontiguousarray(q, dtype=np.uint32)
        qq = qq.reshape(-1, 8) if op == PT_SMUL else qq.reshape(-1, pw)
    out = np.zeros_like(p)
    rc = _fn(curve, "point_op")(op, _ptr(p), _ptr(qq), _ptr(out), p.shape[0])
    if rc != 0:
        raise RuntimeError(f"point_op rc={rc}")
    return out


def gen_scalars(n: int, seed: int = 0, stream: int = 1, dist: int = DIST_UNIFORM, start: int = 0,
                mont: bool = True, threads: int | None = None, curve: int = BN254) -> np.ndarray:
    out = np.zeros((n, 8), dtype=np.uint32)
    _fn(curve, "gen_scalars")(seed, stream, dist, start, n, 1 if mont else 0, _ptr(out), threads or default_threads())
    return out


def gen_points(n: int, seed: int = 0, start: int = 0, threads: int | None = None, curve: int = BN254) -> np.ndarray:
    """P_i = r_i * G, r_i the uniform Fr stream (seed, stream 0)."""
    out = np.zeros((n, _pw(curve)), dtype=np.uint32)
    _fn(curve, "gen_points")(seed, start, n, _ptr(out), threads or default_threads())
    return out


def msm(points: np.ndarray, scalars: np.ndarray, threads: int | None = None, curve: int = BN254) -> np.ndarray:
    """halo2 best_multiexp restated; returns the canonical affine result."""
    pw = _pw(curve)
    points = np.ascontiguousarray(points, dtype=np.uint32).reshape(-1, pw)
    scalars = np.ascontiguousarray(scalars, dtype=np.uint32).reshape(-1, 8)
    n = min(points.shape[0], scalars.shape[0])
    points, scalars = points[:n].copy(), scalars[:n].copy()
    out = np.zeros(pw, dtype=np.uint32)
    _fn(curve, "msm_halo2")(_ptr(points), _ptr(scalars), n, _ptr(out), threads or default_threads())
    return out


def msm_naive(points: np.ndarray, scalars: np.ndarray, curve: int = BN254) -> np.ndarray:
    pw = _pw(curve)
    points = np.ascontiguousarray(points, dtype=np.uint32).reshape(-1, pw)
    scalars = np.ascontiguousarray(scalars, dtype=np.uint32).reshape(-1, 8)
    out = np.zeros(pw, dtype=np.uint32)
    _fn(curve, "msm_naive")(_ptr(points), _ptr(scalars), points.shape[0], _ptr(out))
    return out


def ref_point_op(op: int, p: np.ndarray, q: np.ndarray | None = None, curve: int = BN254) -> np.ndarray:
    """PT_ADD / PT_DBL on affine points through the reference's own
    arithmetic (core/src/common/curve/src/curve_xyzz.cuh)."""
    pw = _pw(curve)
    p = np.ascontiguousarray(p, dtype=np.uint32).reshape(-1, pw)
    out = np.zeros_like(p)
    L = ref_lib()
    add, dbl = (L.ref_point_add, L.ref_point_dbl) if curve == BN254 else (L.ref_bls_point_add, L.ref_bls_point_dbl)
    if op == PT_ADD:
        q = np.ascontiguousarray(q, dtype=np.uint32).reshape(-1, pw)
        add(_ptr(p), _ptr(q), _ptr(out), p.shape[0])
    elif op == PT_DBL:
        dbl(_ptr(p), _ptr(out), p.shape[0])
    else:
        raise ValueError(op)
    return out


def ref_msm_naive(points: np.ndarray, scalars: np.ndarray, curve: int = BN254) -> np.ndarray:
    """Double-and-add MSM through the reference's own host arithmetic."""
    pw = _pw(curve)
    points = np.ascontiguousarray(points, dtype=np.uint32).reshape(-1, pw)
    scalars = np.ascontiguousarray(scalars, dtype=np.uint32).reshape(-1, 8)
    out = np.zeros(pw, dtype=np.uint32)
    fn = ref_lib().ref_msm_naive if curve == BN254 else ref_lib().ref_bls_msm_naive
    fn(_ptr(points), _ptr(scalars), points.shape[0], _ptr(out))
    return out


def precompute(points: np.ndarray, shift: int, n_tables: int, curve: int = BN254) -> np.ndarray:
    """Tables of core/src/msm/src/msm_impl.cuh:358-371: out[j] = 2^(j*shift) * P."""
    pw = _pw(curve)
    points = np.ascontiguousarray(points, dtype=np.uint32).reshape(-1, pw)
    n = points.shape[0]
    out = np.zeros((n_tables, n, pw), dtype=np.uint32)
    _fn(curve, "precompute")(_ptr(points), n, shift, n_tables, _ptr(out))
    return out


# ------------------------------------------------- pure-Python cross-check
# Small affine arithmetic over Python integers (canonical, non-Montgomery),
# used to cross-check the C oracle on tiny inputs.

def py_add(p1, p2, p: int = P):
    if p1 is None:
        return p2
    if p2 is None:
        return p1
    x1, y1 = p1
    x2, y2 = p2
    if x1 == x2:
        if (y1 + y2) % p == 0:
            return None
        lam = 3 * x1 * x1 * pow(2 * y1, -1, p) % p
    else:
        lam = (y2 - y1) * pow(x2 - x1, -1, p) % p
    x3 = (lam * lam - x1 - x2) % p
    return x3, (lam * (x1 - x3) - y1) % p


def py_mul(k: int, pt, p: int = P):
    acc = None
    while k:
        if k & 1:
            acc = py_add(acc, pt, p)
        pt = py_add(pt, pt, p)
        k >>= 1
    return acc


def py_point_from_limbs(a, curve: int = BN254) -> tuple | None:
    _, p, _, w, mr = CURVES[curve]
    a = np.asarray(a, dtype=np.uint32).reshape(2 * w)
    x, y = limbs_to_int(a[:w]), limbs_to_int(a[w:])
    if y == 0:
        return None
    ri = pow(mr, -1, p)
    return x * ri % p, y * ri % p


def py_point_to_limbs(pt, curve: int = BN254) -> np.ndarray:
    _, p, _, w, mr = CURVES[curve]
    if pt is None:
        return np.zeros(2 * w, dtype=np.uint32)
    return np.concatenate([int_to_limbs(pt[0] * mr % p, w), int_to_limbs(pt[1] * mr % p, w)])


def py_msm(points: np.ndarray, scalars: np.ndarray, curve: int = BN254) -> np.ndarray:
    _, p, r, w, _ = CURVES[curve]
    acc = None
    for pt, sc in zip(np.asarray(points).reshape(-1, 2 * w), np.asarray(scalars).reshape(-1, 8)):
        k = from_mont(limbs_to_int(sc), r)
        acc = py_add(acc, py_mul(k, py_point_from_limbs(pt, curve), p), p)
    return py_point_to_limbs(acc, curve)


# ------------------------------------------------------------------- NTT
# The reference's NTT operator (core/src/ntt) over an 8-limb field:
# BN254 Fr (its default NTT_FIELD), BN254 Fq or BLS12-381 Fr.

NTT_FIELDS = {FR: (BN254, 1, R_MOD), FQ: (BN254, 0, P), BLS_FR: (BLS12381, 1, R_BLS)}


def _ntt_fn(field: int, name: str):
    curve, f, _ = NTT_FIELDS[field]
    return _fn(curve, name), f


def root_of_unity(log_n: int, field: int = FR) -> int:
    """A primitive 2^log_n-th root of unity (canonical): g^((m-1)/2^log_n)
    for the least quadratic non-residue g."""
    m = NTT_FIELDS[field][2]
    if (m - 1) % (1 << log_n):
        raise ValueError("2^log_n does not divide m - 1")
    g = 2
    while pow(g, (m - 1) // 2, m) != m - 1:
        g += 1
    w = pow(g, (m - 1) >> log_n, m)
    assert log_n == 0 or pow(w, 1 << (log_n - 1), m) == m - 1
    return w


def mont_limbs(v: int, field: int = FR) -> np.ndarray:
    m = NTT_FIELDS[field][2]
    return int_to_limbs(v * MONT_R % m)


def ntt(x: np.ndarray, unit: np.ndarray, field: int = FR) -> np.ndarray:
    """X[k] = sum_j x[j] unit^(j k), natural order (Montgomery in and out)."""
    x = np.ascontiguousarray(x, dtype=np.uint32).reshape(-1, 8).copy()
    n = x.shape[0]
    log_n = n.bit_length() - 1
    if n != 1 << log_n:
        raise ValueError("length must be a power of two")
    fn, f = _ntt_fn(field, "ntt")
    u = np.ascontiguousarray(unit, dtype=np.uint32).reshape(8)
    rc = fn(f, _ptr(x), log_n, _ptr(u))
    if rc != 0:
        raise RuntimeError(f"ntt rc={rc}")
    return x


def ntt_roots(length: int, unit: np.ndarray, field: int = FR) -> np.ndarray:
    out = np.zeros((length, 8), dtype=np.uint32)
    fn, f = _ntt_fn(field, "ntt_roots")
    fn(f, _ptr(out), length, _ptr(np.ascontiguousarray(unit, dtype=np.uint32).reshape(8)))
    return out


def pq_omegas(pq_deg: int, length: int, unit: np.ndarray, field: int = FR):
    pq = np.zeros(((1 << pq_deg) >> 1, 8), dtype=np.uint32)
    om = np.zeros((32, 8), dtype=np.uint32)
    fn, f = _ntt_fn(field, "pq_omegas")
    rc = fn(f, _ptr(pq), _ptr(om), pq_deg, length, _ptr(np.ascontiguousarray(unit, dtype=np.uint32).reshape(8)))
    if rc != 0:
        raise RuntimeError(f"pq_omegas rc={rc}")
    return pq, om


def distribute_powers(x: np.ndarray, powers: np.ndarray, begin: int = 0, slice_len: int | None = None,
                      poly_len: int | None = None, field: int = FR) -> np.ndarray:
    """x[i] *= powers[((begin + i) % poly_len) % len(powers)]
    (core/src/ntt/src/distribute_powers.cuh:5-11, PolySlice::to_origin)."""
    x = np.ascontiguousarray(x, dtype=np.uint32).reshape(-1, 8)
    powers = np.ascontiguousarray(powers, dtype=np.uint32).reshape(-1, 8)
    n = x.shape[0]
    poly_len = n if poly_len is None else poly_len
    idx = ((begin + np.arange(n, dtype=np.uint64)) % np.uint64(poly_len)) % np.uint64(powers.shape[0])
    return field_op(field, MUL, x, powers[idx.astype(np.int64)])
