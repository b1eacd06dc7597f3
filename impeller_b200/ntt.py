"""Host-side NTT operator over the CUDA C ABI (include/impeller_ntt.h).

Mirrors the reference's Rust operator so that callers (and the tests) read
like the reference's own code:

  - ``SsipNtt``          core/src/ntt.rs:159-208 (in-place NTT, twiddle table
                         of len/2 device elements, asserts power-of-two length)
  - ``SsipPrecompute``   core/src/ntt.rs:211-246 (host twiddle table)
  - ``RecomputeNtt``     core/src/ntt.rs:248-306 (pq + 32 omegas instead of a table)
  - ``GenPqOmegas``      core/src/ntt.rs:308-380 (``get_pq_len`` included)
  - ``DistributePowers`` core/src/ntt.rs:108-157 (optional PolySlice)

Polynomials are torch CUDA tensors of shape (len, 8) int32 (plumbing only):
8 little-endian u32 limbs per element, Montgomery form.  Every transform is
computed by libimpeller_msm.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes
from typing import Callable

import numpy as np

from . import lib as _lib

BN254_FR, BN254_FQ, BLS12381_FR = 0, 1, 2  # IMPELLER_NTT_* (the reference's NTT_FIELD values)
WORDS = 8


def get_stage_threads(field: int = BN254_FR) -> tuple[int, int]:
    """core/src/ntt.rs:383-388: (8, 8) for 32-byte fields."""
    return 8, 8


def _get_deg(deg_stage: int, max_deg_stage: int) -> int:
    """core/src/ntt/src/common.cuh:24-31 (and core/src/ntt.rs:322-339)."""
    rounds = 1
    while True:
        d = deg_stage if rounds == 1 else (deg_stage - 1) // rounds + 1
        if d <= max_deg_stage:
            return d
        rounds += 1


def poly_ptr(t, rotate: int = 0, offset: int = 0, whole_len: int | None = None, length: int | None = None):
    """A PolyPtr over a (whole_len, 8) device tensor: `length` logical
    elements starting at `offset` (or rotated by `rotate`)."""
    whole = t.shape[0] if whole_len is None else whole_len
    n = whole if length is None else length
    return _lib.PolyPtr(t.data_ptr(), n, rotate, offset, whole)


def _stream(stream) -> int | None:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def _host_u32(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a


class SsipNtt:
    """In-place forward NTT of a device polynomial (core/src/ntt.rs:159-208)."""

    def __init__(self, field: int = BN254_FR):
        self.field = field
        self.lib = _lib.load()

    def get_fn(self) -> Callable:
        L = self.lib
        field = self.field

        def f(x, twiddle, stream=None, rotate: int = 0, offset: int = 0, whole_len: int | None = None,
              length: int | None = None) -> None:
            n = x.shape[0] if length is None else length
            assert n & (n - 1) == 0 and n > 0, "length must be a power of two"
            assert twiddle.shape[0] * 2 == n, "twiddle must hold len / 2 elements"
            p = poly_ptr(x, rotate, offset, whole_len, n)
            if field == BN254_FR:
                s1, s2 = get_stage_threads(field)
                rc = L.ssip_ntt(p, twiddle.data_ptr(), n.bit_length() - 1, _stream(stream), s1, s2)
            else:
                rc = L.impeller_ntt(field, p, twiddle.data_ptr(), n.bit_length() - 1, _stream(stream))
            _lib.check(rc, "ssip_ntt")

        return f


class SsipPrecompute:
    """twiddle[i] = unit^i on host arrays (core/src/ntt.rs:211-246)."""

    def __init__(self, field: int = BN254_FR):
        self.field = field
        self.lib = _lib.load()

    def get_fn(self) -> Callable:
        L = self.lib
        field = self.field

        def f(twiddle: np.ndarray, unit: np.ndarray) -> None:
            assert twiddle.shape[0] & (twiddle.shape[0] - 1) == 0, "twiddle length must be a power of two"
            assert twiddle.dtype == np.uint32 and twiddle.flags.c_contiguous
            u = _host_u32(unit).reshape(WORDS)
            if field == BN254_FR:
                rc = L.ssip_precompute(twiddle.ctypes.data, twiddle.shape[0], u.ctypes.data)
            else:
                rc = L.impeller_ntt_precompute(field, twiddle.ctypes.data, twiddle.shape[0], u.ctypes.data)
            _lib.check(rc, "ssip_precompute")

        return f


class RecomputeNtt:
    """In-place NTT with recomputed twiddles (core/src/ntt.rs:248-306)."""

    def __init__(self, field: int = BN254_FR):
        self.field = field
        self.lib = _lib.load()

    def get_fn(self) -> Callable:
        L = self.lib
        field = self.field

        def f(x, pq, omegas, stream=None, rotate: int = 0, offset: int = 0, whole_len: int | None = None,
              length: int | None = None) -> None:
            n = x.shape[0] if length is None else length
            assert n & (n - 1) == 0 and n > 0, "length must be a power of two"
            assert pq.shape[0] & (pq.shape[0] - 1) == 0, "pq length must be a power of two"
            assert omegas.shape[0] == 32
            pq_deg = (pq.shape[0] - 1).bit_length() + 1 if pq.shape[0] > 1 else 1
            p = poly_ptr(x, rotate, offset, whole_len, n)
            if field == BN254_FR:
                s1, s2 = get_stage_threads(field)
                rc = L.recompute_ntt(p, pq.data_ptr(), pq_deg, omegas.data_ptr(), n.bit_length() - 1,
                                     _stream(stream), s1, s2)
            else:
                rc = L.impeller_ntt_recompute(field, p, omegas.data_ptr(), n.bit_length() - 1, _stream(stream))
            _lib.check(rc, "recompute_ntt")

        return f


class GenPqOmegas:
    """Host pq / omegas tables for RecomputeNtt (core/src/ntt.rs:308-380)."""

    def __init__(self, field: int = BN254_FR):
        self.field = field
        self.lib = _lib.load()

    def get_pq_len(self, log_len: int) -> int:
        s1, s2 = get_stage_threads(self.field)
        deg1 = _get_deg((log_len + 1) // 2, s1 + 1)
        deg2 = _get_deg(log_len // 2, (s2 + 2) // 2)
        return 1 << (max(deg1, deg2) - 1)

    def get_fn(self) -> Callable:
        L = self.lib
        field = self.field

        def f(pq: np.ndarray, omegas: np.ndarray, length: int, unit: np.ndarray) -> None:
            assert omegas.shape[0] == 32
            pq_deg = (pq.shape[0] - 1).bit_length() + 1 if pq.shape[0] > 1 else 1
            u = _host_u32(unit).reshape(WORDS)
            if field == BN254_FR:
                L.gen_pq_omegas(pq.ctypes.data, omegas.ctypes.data, pq_deg, length, u.ctypes.data)
            else:
                _lib.check(L.impeller_ntt_gen_pq_omegas(field, pq.ctypes.data, omegas.ctypes.data, pq_deg, length,
                                                        u.ctypes.data), "gen_pq_omegas")

        return f


class DistributePowers:
    """x[i] *= powers[slice.to_origin(i) mod len(powers)] (core/src/ntt.rs:108-157)."""

    def __init__(self, field: int = BN254_FR):
        self.field = field
        self.lib = _lib.load()

    def get_fn(self) -> Callable:
        L = self.lib
        field = self.field

        def f(x, powers, stream=None, poly_slice: tuple | None = None, rotate: int = 0, offset: int = 0,
              whole_len: int | None = None, length: int | None = None) -> None:
            n = x.shape[0] if length is None else length
            sl = _lib.PolySlice(*(poly_slice if poly_slice is not None else (0, n, n)))
            p = poly_ptr(x, rotate, offset, whole_len, n)
            if field == BN254_FR:
                rc = L.distribute_powers(p, powers.data_ptr(), powers.shape[0], _stream(stream), ctypes.byref(sl))
            else:
                rc = L.impeller_ntt_distribute_powers(field, p, powers.data_ptr(), powers.shape[0], _stream(stream),
                                                      ctypes.byref(sl))
            _lib.check(rc, "distribute_powers")

        return f


def launches(log_len: int) -> int:
    """Kernel launches of one transform of 2^log_len elements."""
    return int(_lib.load().impeller_ntt_launches(log_len))


# ---------------------------------------------------------------- helpers

MODULI = {
    BN254_FR: 21888242871839275222246405745257275088548364400416034343698204186575808495617,
    BN254_FQ: 21888242871839275222246405745257275088696311157297823662689037894645226208583,
    BLS12381_FR: 0x73eda753299d7d483339d80809a1d80553bda402fffe5bfeffffffff00000001,
}


def root_of_unity(log_n: int, field: int = BN254_FR) -> int:
    """A primitive 2^log_n-th root of unity of the field (canonical integer):
    g^((m - 1) / 2^log_n) for the least quadratic non-residue g."""
    m = MODULI[field]
    if (m - 1) % (1 << log_n):
        raise ValueError(f"the field has no 2^{log_n}-th roots of unity")
    g = 2
    while pow(g, (m - 1) // 2, m) != m - 1:
        g += 1
    return pow(g, (m - 1) >> log_n, m)


def to_mont_limbs(v: int, field: int = BN254_FR) -> np.ndarray:
    """v (canonical) as 8 u32 Montgomery limbs (R = 2^256)."""
    x = v * (1 << 256) % MODULI[field]
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(WORDS)], dtype=np.uint32)


def butterfly_products(log_n: int) -> int:
    """Montgomery products one transform of 2^log_n elements makes: every
    radix-2 butterfly multiplies by its twiddle except where the twiddle is
    w^0 (n/2^(s+1) butterflies of stage s), i.e. n (log_n / 2 - 1) + 1."""
    n = 1 << log_n
    return sum(n // 2 - n // (2 << s) for s in range(log_n))


if __name__ == "__main__":
    # Profiling driver: python -m impeller_b200.ntt [log_n] [steps] [recompute]
    # (one twiddle precompute, three warm-up transforms, then `steps` more).
    import sys

    import torch

    from . import msm as _msm
    log_n = int(sys.argv[1]) if len(sys.argv) > 1 else 24
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else 3
    recompute = len(sys.argv) > 3 and sys.argv[3] == "recompute"
    n = 1 << log_n
    x = _msm.gen_scalars_device(n, seed=7, stream_id=11)
    unit = to_mont_limbs(root_of_unity(log_n))
    if recompute:
        g = GenPqOmegas()
        pq = np.zeros((g.get_pq_len(log_n), WORDS), np.uint32)
        om = np.zeros((32, WORDS), np.uint32)
        g.get_fn()(pq, om, n, unit)
        d_pq, d_om = (torch.from_numpy(a.view(np.int32)).cuda() for a in (pq, om))
        f = RecomputeNtt().get_fn()
        run = lambda: f(x, d_pq, d_om)  # noqa: E731
    else:
        tw = np.zeros((n // 2, WORDS), np.uint32)
        SsipPrecompute().get_fn()(tw, unit)
        d_tw = torch.from_numpy(tw.view(np.int32)).cuda()
        f = SsipNtt().get_fn()
        run = lambda: f(x, d_tw)  # noqa: E731
    for _ in range(3 + steps):
        run()
    torch.cuda.synchronize()
    print(f"{3 + steps} transforms of 2^{log_n} done")
