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

FQ, FR = 0, 1
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
        L.orc_field_op.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, _u32p, _u32p, ctypes.c_uint64]
        L.orc_point_op.argtypes = [ctypes.c_int, _u32p, _u32p, _u32p, ctypes.c_uint64]
        L.orc_gen_scalars.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64,
                                      ctypes.c_uint64, ctypes.c_int, _u32p, ctypes.c_int]
        L.orc_gen_points.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, _u32p, ctypes.c_int]
        L.orc_msm_halo2.argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p, ctypes.c_int]
        L.orc_msm_naive.argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p]
        L.orc_precompute.argtypes = [_u32p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, _u32p]
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

def field_op(field: int, op: int, a: np.ndarray, b: np.ndarray | None = None, use_ref: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint32).reshape(-1, 8)
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.uint32).reshape(-1, 8)
    out = np.zeros_like(a)
    L = ref_lib() if use_ref else lib()
    fn = L.ref_field_op if use_ref else L.orc_field_op
    rc = fn(field, op, _ptr(a), _ptr(bb), _ptr(out), a.shape[0])
    if rc != 0:
        raise RuntimeError(f"field_op rc={rc}")
    return out


def point_op(op: int, p: np.ndarray, q: np.ndarray | None = None) -> np.ndarray:
    p = np.ascontiguousarray(p, dtype=np.uint32).reshape(-1, 16)
    qq = None
    if q is not None:
        qq = np.ascontiguousarray(q, dtype=np.uint32)
        qq = qq.reshape(-1, 8) if op == PT_SMUL else qq.reshape(-1, 16)
    out = np.zeros_like(p)
    rc = lib().orc_point_op(op, _ptr(p), _ptr(qq), _ptr(out), p.shape[0])
    if rc != 0:
        raise RuntimeError(f"point_op rc={rc}")
    return out


def gen_scalars(n: int, seed: int = 0, stream: int = 1, dist: int = DIST_UNIFORM, start: int = 0,
                mont: bool = True, threads: int | None = None) -> np.ndarray:
    out = np.zeros((n, 8), dtype=np.uint32)
    lib().orc_gen_scalars(seed, stream, dist, start, n, 1 if mont else 0, _ptr(out),
                          threads or default_threads())
    return out


def gen_points(n: int, seed: int = 0, start: int = 0, threads: int | None = None) -> np.ndarray:
    """P_i = r_i * G, r_i the uniform Fr stream (seed, stream 0)."""
    out = np.zeros((n, 16), dtype=np.uint32)
    lib().orc_gen_points(seed, start, n, _ptr(out), threads or default_threads())
    return out


def msm(points: np.ndarray, scalars: np.ndarray, threads: int | None = None) -> np.ndarray:
    """halo2 best_multiexp restated; returns the canonical affine result (16 u32)."""
    points = np.ascontiguousarray(points, dtype=np.uint32).reshape(-1, 16)
    scalars = np.ascontiguousarray(scalars, dtype=np.uint32).reshape(-1, 8)
    n = min(points.shape[0], scalars.shape[0])
    points, scalars = points[:n].copy(), scalars[:n].copy()
    out = np.zeros(16, dtype=np.uint32)
    lib().orc_msm_halo2(_ptr(points), _ptr(scalars), n, _ptr(out), threads or default_threads())
    return out


def msm_naive(points: np.ndarray, scalars: np.ndarray) -> np.ndarray:
    points = np.ascontiguousarray(points, dtype=np.uint32).reshape(-1, 16)
    scalars = np.ascontiguousarray(scalars, dtype=np.uint32).reshape(-1, 8)
    out = np.zeros(16, dtype=np.uint32)
    lib().orc_msm_naive(_ptr(points), _ptr(scalars), points.shape[0], _ptr(out))
    return out


def ref_msm_naive(points: np.ndarray, scalars: np.ndarray) -> np.ndarray:
    points = np.ascontiguousarray(points, dtype=np.uint32).reshape(-1, 16)
    scalars = np.ascontiguousarray(scalars, dtype=np.uint32).reshape(-1, 8)
    out = np.zeros(16, dtype=np.uint32)
    ref_lib().ref_msm_naive(_ptr(points), _ptr(scalars), points.shape[0], _ptr(out))
    return out


def precompute(points: np.ndarray, shift: int, n_tables: int) -> np.ndarray:
    """Tables of core/src/msm/src/msm_impl.cuh:358-371: out[j] = 2^(j*shift) * P."""
    points = np.ascontiguousarray(points, dtype=np.uint32).reshape(-1, 16)
    n = points.shape[0]
    out = np.zeros((n_tables, n, 16), dtype=np.uint32)
    lib().orc_precompute(_ptr(points), n, shift, n_tables, _ptr(out))
    return out


# ------------------------------------------------- pure-Python cross-check
# Small affine arithmetic over Python integers (canonical, non-Montgomery),
# used to cross-check the C oracle on tiny inputs.

def py_add(p1, p2):
    if p1 is None:
        return p2
    if p2 is None:
        return p1
    x1, y1 = p1
    x2, y2 = p2
    if x1 == x2:
        if (y1 + y2) % P == 0:
            return None
        lam = 3 * x1 * x1 * pow(2 * y1, -1, P) % P
    else:
        lam = (y2 - y1) * pow(x2 - x1, -1, P) % P
    x3 = (lam * lam - x1 - x2) % P
    return x3, (lam * (x1 - x3) - y1) % P


def py_mul(k: int, p):
    acc = None
    while k:
        if k & 1:
            acc = py_add(acc, p)
        p = py_add(p, p)
        k >>= 1
    return acc


def py_point_from_limbs(a) -> tuple | None:
    a = np.asarray(a, dtype=np.uint32).reshape(16)
    x, y = limbs_to_int(a[:8]), limbs_to_int(a[8:])
    if y == 0:
        return None
    return from_mont(x, P), from_mont(y, P)


def py_point_to_limbs(p) -> np.ndarray:
    if p is None:
        return np.zeros(16, dtype=np.uint32)
    return np.concatenate([int_to_limbs(to_mont(p[0], P)), int_to_limbs(to_mont(p[1], P))])


def py_msm(points: np.ndarray, scalars: np.ndarray) -> np.ndarray:
    acc = None
    for pt, s in zip(np.asarray(points).reshape(-1, 16), np.asarray(scalars).reshape(-1, 8)):
        k = from_mont(limbs_to_int(s), R_MOD)
        acc = py_add(acc, py_mul(k, py_point_from_limbs(pt)))
    return py_point_to_limbs(acc)
