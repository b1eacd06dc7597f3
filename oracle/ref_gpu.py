"""The reference's own GPU MSM, compiled for sm_100a (test and measurement
infrastructure only).

``_ref/libref_msm_<curve>_<c>_<alpha>_false.so`` is the reference's
``core/src/msm/src/msm.cu`` built unmodified from its source tree by
``oracle/Makefile`` (target ``ref_gpu``), one library per (curve, window
size, target window) exactly as the reference's ``Makefile.msm`` builds one
per configuration (curve ``bn254`` or ``bls12381``).  This module drives it through its C ABI
(``core/src/msm/src/msm.h:4-11``) the way the reference's Rust operator does
(``core/src/msm.rs:169-190, 282-366``; ``core/tests/msm.rs:150-240``):

* a size query with ``buffers = NULL`` for the per-card scratch size;
* one caller-allocated device buffer per card;
* ``msm_precompute`` filling tables 1.. of pinned host point arrays from
  table 0, once;
* blocking ``msm`` calls on pinned host points and scalars (Montgomery form),
  affine results (16 u32 on BN254, 24 on BLS12-381).

Only ``tests/`` (as a second parity pin, against the reference's real GPU
output) and ``bench.py --impl reference`` (as the reference's B200 timing)
use it.  The library exists only where the reference sources were present at
build time; ``available()`` says whether it was built.
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

LAMBDA = 254  # BN254 scalar bits (MSM_BITS)
BN254, BLS12381 = 0, 1
CURVE_NAMES = {BN254: "bn254", BLS12381: "bls12381"}
CURVE_BITS = {BN254: 254, BLS12381: 255}  # MSM_BITS
POINT_WORDS = {BN254: 16, BLS12381: 24}

# (window size, target window): MsmConfig::default() and the reference cost
# model's choice for n = 2^22 (core/src/msm/tuning/cost_model.py
# --k=22 --n=1 --l=254 --p=254 prints alpha 8, s 17, w 16, h 1).
DEFAULT_CONFIG = (16, 16)
TUNED_2E22_CONFIG = (17, 8)
TUNED_2E22_PARTS = 16


def lib_path(c: int, alpha: int, curve: int = BN254) -> str:
    return os.path.join(HERE, "_ref", f"libref_msm_{CURVE_NAMES[curve]}_{c}_{alpha}_false.so")


def available(c: int = DEFAULT_CONFIG[0], alpha: int = DEFAULT_CONFIG[1], curve: int = BN254) -> bool:
    return os.path.exists(lib_path(c, alpha, curve))


def n_precompute(c: int, alpha: int, curve: int = BN254) -> int:
    """MsmConfig::get_precompute (common/src/msm_config.rs:17-25)."""
    actual = -(-CURVE_BITS[curve] // c)
    n_windows = min(actual, alpha)
    return -(-actual // n_windows)


def _pinned_u32(shape):
    import torch
    t = torch.empty(int(np.prod(shape)), dtype=torch.int32, pin_memory=True)
    return t, t.numpy().view(np.uint32).reshape(shape)


class RefGpuMsm:
    """One reference MSM configuration over an n-point SRS held in pinned
    host memory (tables 1.. precomputed by the reference on the GPU)."""

    def __init__(self, points: np.ndarray, c: int = DEFAULT_CONFIG[0], alpha: int = DEFAULT_CONFIG[1],
                 parts: int = 1, device: int = 0, curve: int = BN254):
        import torch
        path = lib_path(c, alpha, curve)
        self.pw = pw = POINT_WORDS[curve]
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle ref_gpu needs the reference sources)")
        self.lib = ctypes.CDLL(path)
        u32p, u32pp = ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32))
        self.lib.msm.restype = ctypes.c_int
        self.lib.msm.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_ulong),
                                 ctypes.c_ulonglong, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                                 ctypes.c_uint, u32p, u32pp, ctypes.c_uint, u32pp, u32pp]
        self.lib.msm_precompute.restype = ctypes.c_int
        self.lib.msm_precompute.argtypes = [ctypes.c_ulonglong, u32pp, ctypes.c_uint]
        points = np.ascontiguousarray(points, dtype=np.uint32).reshape(-1, pw)
        self.n = points.shape[0]
        self.c, self.alpha, self.parts = c, alpha, parts
        # get_best_config: one scalar and one point stage for a single part, two otherwise
        self.stages = 1 if parts == 1 else 2
        self.device = device
        self.cards = (ctypes.c_uint32 * 1)(device)
        self.k = n_precompute(c, alpha, curve)
        self._tables = []
        ptrs = []
        for j in range(self.k):
            t, a = _pinned_u32((self.n, pw))
            if j == 0:
                a[:] = points
            self._tables.append((t, a))
            ptrs.append(a.ctypes.data_as(u32p))
        self.h_points = (u32p * self.k)(*ptrs)
        if self.k > 1:
            rc = self.lib.msm_precompute(self.n, self.h_points, 1)
            if rc != 0:
                raise RuntimeError(f"reference msm_precompute failed: cudaError {rc}")
        size = (ctypes.c_ulong * 1)()
        rc = self.lib.msm(None, size, self.n, 1, parts, self.stages, self.stages, 1, self.cards,
                          None, 0, None, None)
        if rc != 0:
            raise RuntimeError(f"reference msm size query failed: cudaError {rc}")
        self.buffer_bytes = int(size[0])
        self._buf = torch.empty(self.buffer_bytes, dtype=torch.uint8, device=f"cuda:{device}")
        self.buffers = (ctypes.c_void_p * 1)(self._buf.data_ptr())
        self._scal_t, self._scal = _pinned_u32((self.n, 8))
        self._res_t, self._res = _pinned_u32((pw,))

    def tables(self) -> np.ndarray:
        """The host point tables after the reference's precompute (k x n x point words)."""
        return np.stack([a for _, a in self._tables])

    def load_scalars(self, scalars: np.ndarray) -> None:
        self._scal[:] = np.ascontiguousarray(scalars, dtype=np.uint32).reshape(-1, 8)[: self.n]

    def run(self) -> np.ndarray:
        """One blocking reference MSM over the loaded scalars; the affine result."""
        u32p = ctypes.POINTER(ctypes.c_uint32)
        scal = (u32p * 1)(self._scal.ctypes.data_as(u32p))
        res = (u32p * 1)(self._res.ctypes.data_as(u32p))
        size = (ctypes.c_ulong * 1)(self.buffer_bytes)
        rc = self.lib.msm(self.buffers, size, self.n, 1, self.parts, self.stages, self.stages, 1, self.cards,
                          self.h_points, 1, scal, res)
        if rc != 0:
            raise RuntimeError(f"reference msm failed: cudaError {rc}")
        return self._res.copy()

    def msm(self, scalars: np.ndarray) -> np.ndarray:
        self.load_scalars(scalars)
        return self.run()

    def time_calls(self, scalar_sets, warmup: int, steps: int) -> float:
        """Mean wall time (ms) of blocking calls, host buffers in and out: the
        call returns only after its result is on the host."""
        for w in range(warmup):
            self.msm(scalar_sets[w % len(scalar_sets)])
        total = 0.0
        for k in range(steps):
            self.load_scalars(scalar_sets[k % len(scalar_sets)])
            t0 = time.perf_counter()
            self.run()
            total += time.perf_counter() - t0
        return total / steps * 1e3

    def close(self) -> None:
        self._buf = None
        self._tables = []
