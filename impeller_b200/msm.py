"""Host-side MSM operator over the CUDA C ABI.

Mirrors the reference's operator so that callers (and the tests) read like
the reference's own code:

  - ``MsmConfig``       common/src/msm_config.rs:4-56
  - ``get_best_config`` core/src/msm.rs:36-99 (autotune table instead of the
                        cost_model.py subprocess)
  - ``MSM``             core/src/msm.rs:114-135, 260-373 (library by name,
                        get_buffer_size, the FuncCall closure of get_fn)
  - ``MSMPrecompute``   core/src/msm.rs:137-191

and adds the B200 entry points the reference has no counterpart for: a
resident-SRS ``MsmContext`` with single and batched (CUDA-graph) MSMs.

Device memory is plain torch CUDA tensors (plumbing only); every MSM is
computed by libimpeller_msm.so.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from . import lib as _lib

BN254_BITS = 254

# Curves (include/impeller_msm.h IMPELLER_CURVE_*): the reference's MSM
# library list covers bn254 (254-bit scalars) and bls12381 (255-bit scalars,
# 381-bit base field), core/src/msm/xmake.lua and core/src/msm.rs:24-34.
BN254, BLS12381 = 0, 1
CURVE_NAMES = {BN254: "bn254", BLS12381: "bls12381"}
SCALAR_BITS = {BN254: 254, BLS12381: 255}
POINT_WORDS = {BN254: 16, BLS12381: 24}  # affine point, u32 words


def _u32pp(arrays: Sequence[np.ndarray]):
    arr = (_lib.c_u32p * len(arrays))()
    for i, a in enumerate(arrays):
        arr[i] = a.ctypes.data_as(_lib.c_u32p) if a is not None else None
    return arr


# ------------------------------------------------------------------ config

@dataclass
class MsmConfig:
    """common/src/msm_config.rs:4-14."""
    window_size: int = 16
    target_window: int = 16
    cards: list = field(default_factory=lambda: [0])
    debug: bool = False
    batch_per_run: int = 1
    parts: int = 1
    stage_scalars: int = 1
    stage_points: int = 1
    bits: int | None = None  # scalar bits; None -> the curve's
    curve: int = BN254

    def __post_init__(self):
        if self.curve not in CURVE_NAMES:
            raise ValueError(f"unknown curve {self.curve}")
        if self.bits is None:
            self.bits = SCALAR_BITS[self.curve]

    def get_precompute(self) -> int:
        """common/src/msm_config.rs:17-25."""
        actual = -(-self.bits // self.window_size)
        n_windows = actual if actual < self.target_window else self.target_window
        return -(-actual // n_windows)


def lib_name(config: MsmConfig) -> str:
    """core/src/msm.rs:101-112: msm_{curve}_{window}_{target}_{debug}."""
    return (f"msm_{CURVE_NAMES[config.curve]}_{config.window_size}_{config.target_window}_"
            f"{'true' if config.debug else 'false'}")


_shims: dict[str, ctypes.CDLL] = {}


def load_msm_library(config: MsmConfig) -> ctypes.CDLL:
    """The library exporting msm / msm_precompute for this configuration.

    Like core/src/msm.rs:260-280 (make the .so on first use, then load it by
    name): lib/lib{lib_name}.so is a small shim that forwards to
    libimpeller_msm.so with the window size and target window baked in."""
    name = lib_name(config)
    if name in _shims:
        return _shims[name]
    core = _lib.load()  # the shim resolves impeller_msm_cfg from here
    from . import build as _build
    path = _build.build_shim(config.window_size, config.target_window, config.debug, config.curve)
    L = ctypes.CDLL(path)
    for sym in ("msm", "msm_precompute"):
        fn = getattr(L, sym)
        fn.restype, fn.argtypes = _lib.SIGNATURES[sym]
    _shims[name] = L
    del core
    return L


def get_best_config(length: int, batches: int, mem_limit: int, cards: Sequence[int] = (0,),
                    curve: int = BN254) -> MsmConfig:
    """core/src/msm.rs:36-99: pick (window, target window, parts,
    batch_per_run) for `batches` MSMs of `length` points under `mem_limit`
    bytes of device memory.  The window comes from the autotune table; no
    window tables (target_window = number of windows); the largest
    batch_per_run and the fewest parts whose scratch fits."""
    L = _lib.load()
    c = int(L.impeller_default_window_curve(max(1, length), curve))
    W = window_count(c, curve)
    parts = 1
    while True:
        for bpr in range(min(batches, 8), 0, -1):
            cfg = MsmConfig(window_size=c, target_window=W, cards=list(cards), batch_per_run=bpr, parts=parts,
                            stage_scalars=1 if parts == 1 else 2, stage_points=1 if parts == 1 else 2,
                            curve=curve)
            if max(MSM(cfg).get_buffer_size(length)) <= mem_limit:
                return cfg
        parts *= 2
        if parts > max(1, length):
            raise ValueError("no configuration fits the memory limit")


# ------------------------------------------------------- runtime variables
# Minimal stand-ins for the runtime's Variable kinds the MSM FuncCall takes
# (runtime/src/args.rs): host point and scalar arrays, a GPU buffer, a result.

@dataclass
class PointArray:
    values: np.ndarray  # (len, POINT_WORDS[curve]) uint32

    @property
    def len(self) -> int:
        return self.values.shape[0]


@dataclass
class ScalarArray:
    values: np.ndarray  # (len, 8) uint32, Montgomery Fr
    rotation: int = 0

    def get_rotation(self) -> int:
        return self.rotation


@dataclass
class GpuBuffer:
    ptr: int
    size: int
    device: int = 0


@dataclass
class Point:
    value: np.ndarray = field(default_factory=lambda: np.zeros(16, dtype=np.uint32))  # resized to the curve's


def alloc_gpu_buffer(size: int, device: int = 0):
    """A device buffer for the MSM scratch (torch allocator, plumbing)."""
    import torch
    t = torch.empty(max(size, 1), dtype=torch.uint8, device=f"cuda:{device}")
    return GpuBuffer(ptr=t.data_ptr(), size=size, device=device), t


class MSM:
    """core/src/msm.rs:114-135 and the RegisteredFunction impl at :305-373."""

    def __init__(self, config: MsmConfig, library: ctypes.CDLL | None = None):
        self.config = config
        if library is not None:
            self.lib = library
        elif (config.window_size == 16 and config.target_window == 16 and not config.debug
              and config.curve == BN254):
            self.lib = _lib.load()  # the default symbols of the core library
        else:
            self.lib = load_msm_library(config)

    def get_buffer_size(self, length: int) -> list:
        """core/src/msm.rs:282-302: buffers == NULL returns per-card sizes."""
        cfg = self.config
        sizes = (ctypes.c_ulong * len(cfg.cards))()
        cards = (ctypes.c_uint * len(cfg.cards))(*cfg.cards)
        rc = self.lib.msm(None, sizes, length, cfg.batch_per_run, cfg.parts, cfg.stage_scalars, cfg.stage_points,
                          len(cfg.cards), cards, None, 0, None, None)
        _lib.check(rc, "msm (size query)")
        return list(sizes)

    def get_fn(self) -> Callable:
        """The FuncCall closure (core/src/msm.rs:311-366).

        f(mut_var, var, gpu_mapping): var = [PointArray x n_precompute,
        ScalarArray x batches]; mut_var = [GpuBuffer x cards, Point x batches]."""
        cfg = self.config
        n_precompute = cfg.get_precompute()
        c_func = self.lib.msm

        def f(mut_var: list, var: list, gpu_mapping: Callable[[int], int] = lambda x: x, _slice=None) -> None:
            batches = len(var) - n_precompute
            assert len(mut_var) == batches + len(cfg.cards)
            length = var[0].len
            h_points = [np.ascontiguousarray(var[i].values, dtype=np.uint32) for i in range(n_precompute)]
            h_scalars = []
            for v in var[n_precompute:]:
                assert v.get_rotation() == 0, "currently, we don't support rotate in msm"
                h_scalars.append(np.ascontiguousarray(v.values, dtype=np.uint32))
            buffers, answers = mut_var[:len(cfg.cards)], mut_var[len(cfg.cards):]
            bufs = (ctypes.c_void_p * len(buffers))(*[b.ptr for b in buffers])
            results = [np.zeros(POINT_WORDS[cfg.curve], dtype=np.uint32) for _ in answers]
            cards = [gpu_mapping(c) for c in cfg.cards]
            rc = c_func(bufs, None, length, cfg.batch_per_run, cfg.parts, cfg.stage_scalars, cfg.stage_points,
                        len(cards), (ctypes.c_uint * len(cards))(*cards), _u32pp(h_points), batches,
                        _u32pp(h_scalars), _u32pp(results))
            _lib.check(rc, "msm")
            for a, r in zip(answers, results):
                a.value = r

        return f

    def run(self, points_tables: Sequence[np.ndarray], scalars: Sequence[np.ndarray],
            buffers: Sequence[GpuBuffer]) -> list:
        """Convenience: marshal like the runtime does and return the results."""
        var = [PointArray(np.asarray(p)) for p in points_tables] + [ScalarArray(np.asarray(s)) for s in scalars]
        answers = [Point() for _ in scalars]
        self.get_fn()(list(buffers) + answers, var)
        return [a.value for a in answers]


class MSMPrecompute:
    """core/src/msm.rs:137-191."""

    def __init__(self, config: MsmConfig, library: ctypes.CDLL | None = None):
        self.config = config
        if library is not None:
            self.lib = library
        elif (config.window_size == 16 and config.target_window == 16 and not config.debug
              and config.curve == BN254):
            self.lib = _lib.load()
        else:
            self.lib = load_msm_library(config)

    def get_fn(self) -> Callable:
        c_func = self.lib.msm_precompute

        def f(target: list, length: int, max_cards: int) -> None:
            arrays = [np.ascontiguousarray(t.values if isinstance(t, PointArray) else t, dtype=np.uint32)
                      for t in target]
            rc = c_func(length, _u32pp(arrays), max_cards)
            _lib.check(rc, "msm_precompute")
            for t, a in zip(target, arrays):
                if isinstance(t, PointArray):
                    t.values = a
                elif isinstance(t, np.ndarray) and t is not a:
                    t[...] = a.reshape(t.shape)

        return f


# ---------------------------------------------------- device plumbing (torch)

def to_device(a: np.ndarray, device: int = 0):
    import torch
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return torch.from_numpy(a.view(np.int32)).to(f"cuda:{device}")


def to_host(t) -> np.ndarray:
    return t.detach().cpu().numpy().view(np.uint32)


def _stream_handle(stream) -> int | None:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def gen_points_device(n: int, seed: int = 0, start: int = 0, device: int = 0, stream=None, curve: int = BN254):
    import torch
    out = torch.empty((n, POINT_WORDS[curve]), dtype=torch.int32, device=f"cuda:{device}")
    _lib.check(_lib.load().impeller_gen_points_curve(curve, out.data_ptr(), n, seed, start, _stream_handle(stream)),
               "impeller_gen_points")
    return out


def gen_scalars_device(n: int, seed: int = 0, stream_id: int = 1, dist: int = 0, start: int = 0, mont: bool = True,
                       device: int = 0, stream=None, curve: int = BN254):
    import torch
    out = torch.empty((n, 8), dtype=torch.int32, device=f"cuda:{device}")
    _lib.check(_lib.load().impeller_gen_scalars_curve(curve, out.data_ptr(), n, seed, stream_id, dist, start,
                                                      1 if mont else 0, _stream_handle(stream)),
               "impeller_gen_scalars")
    return out


def set_window_table(table: dict) -> None:
    """Load an autotune table {log2 n: c or (c, tables_c)} into the library;
    an empty dict selects the built-in cost model."""
    keys = sorted(table)
    cnt = len(keys)
    vals = [table[k] if isinstance(table[k], tuple) else (table[k], 0) for k in keys]
    lg = (ctypes.c_uint32 * cnt)(*keys)
    cs = (ctypes.c_uint32 * cnt)(*[int(v[0]) for v in vals])
    ct = (ctypes.c_uint32 * cnt)(*[int(v[1]) for v in vals])
    _lib.check(_lib.load().impeller_set_window_table(lg, cs, ct, cnt), "impeller_set_window_table")


def restore_default_window_table() -> None:
    """Reinstall the measured table compiled into the library."""
    from . import autotune
    if not autotune.load_table():
        set_window_table({})


def default_window(n: int, curve: int = BN254) -> int:
    return int(_lib.load().impeller_default_window_curve(n, curve))


def table_window(n: int) -> int:
    return int(_lib.load().impeller_table_window(n))


# --------------------------------------------------- resident-SRS context

class MsmContext:
    """Points uploaded once and kept in HBM; MSMs over prefixes of them."""

    def __init__(self, points, device: int = 0, curve: int = BN254):
        L = _lib.load()
        self.device = device
        self.curve = curve
        self.pw = POINT_WORDS[curve]
        h = ctypes.c_void_p()
        if hasattr(points, "data_ptr"):
            self._points_ref = points  # borrowed device tensor, keep alive
            n = points.numel() // self.pw
            _lib.check(L.impeller_ctx_create_curve(ctypes.byref(h), device, points.data_ptr(), n, 1, curve),
                       "impeller_ctx_create")
        else:
            pts = np.ascontiguousarray(points, dtype=np.uint32)
            n = pts.size // self.pw
            _lib.check(L.impeller_ctx_create_curve(ctypes.byref(h), device, pts.ctypes.data, n, 0, curve),
                       "impeller_ctx_create")
        self.handle = h
        self.len = n

    def precompute(self, c: int) -> None:
        """Keep W(c) window tables (2^(j*c) * P) resident for window c."""
        _lib.check(_lib.load().impeller_ctx_precompute(self.handle, c), "impeller_ctx_precompute")

    def window(self, n: int) -> int:
        return int(_lib.load().impeller_ctx_window(self.handle, n))

    def launches(self, n: int, c: int = 0) -> int:
        """Kernel launches of one MSM of n points with window c (0: the context's)."""
        return int(_lib.load().impeller_ctx_launches(self.handle, n, c))

    def close(self) -> None:
        if self.handle:
            _lib.load().impeller_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def msm_device(self, d_scalars, n: int | None = None, c: int = 0, out=None, stream=None):
        import torch
        n = d_scalars.shape[0] if n is None else n
        if out is None:
            out = torch.empty(self.pw, dtype=torch.int32, device=f"cuda:{self.device}")
        _lib.check(_lib.load().impeller_msm_device(self.handle, d_scalars.data_ptr(), n, c, out.data_ptr(),
                                                   _stream_handle(stream)), "impeller_msm_device")
        return out

    def msm_host(self, h_scalars: np.ndarray, c: int = 0, stream=None) -> np.ndarray:
        sc = np.ascontiguousarray(h_scalars, dtype=np.uint32)
        out = np.zeros(self.pw, dtype=np.uint32)
        _lib.check(_lib.load().impeller_msm_host(self.handle, sc.ctypes.data, sc.shape[0], c, out.ctypes.data,
                                                 _stream_handle(stream)), "impeller_msm_host")
        return out

    def batch(self, sizes: Sequence[int], windows: Sequence[int] | None = None, graph: bool = True) -> "MsmBatch":
        return MsmBatch(self, sizes, windows, graph)


class MsmBatch:
    """Many MSMs of uneven sizes in one plan; one launch per phase, optionally
    replayed from a CUDA graph."""

    def __init__(self, ctx: MsmContext, sizes: Sequence[int], windows: Sequence[int] | None, graph: bool):
        L = _lib.load()
        self.ctx = ctx
        self.sizes = [int(s) for s in sizes]
        cnt = len(self.sizes)
        sz = (ctypes.c_uint64 * cnt)(*self.sizes)
        ws = (ctypes.c_uint * cnt)(*(windows or [0] * cnt))
        h = ctypes.c_void_p()
        _lib.check(L.impeller_batch_create(ctypes.byref(h), ctx.handle, sz, ws, cnt, 1 if graph else 0),
                   "impeller_batch_create")
        self.handle = h

    @property
    def launches(self) -> int:
        return int(_lib.load().impeller_batch_launches(self.handle))

    def run(self, d_scalars: Sequence, out=None, stream=None):
        import torch
        cnt = len(self.sizes)
        if out is None:
            out = torch.empty((cnt, self.ctx.pw), dtype=torch.int32, device=f"cuda:{self.ctx.device}")
        ptrs = (ctypes.c_void_p * cnt)(*[s.data_ptr() for s in d_scalars])
        _lib.check(_lib.load().impeller_batch_run(self.handle, ptrs, out.data_ptr(), _stream_handle(stream)),
                   "impeller_batch_run")
        return out

    def close(self) -> None:
        if self.handle:
            _lib.load().impeller_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def n_precompute(window_size: int, target_window: int, curve: int = BN254) -> int:
    return int(_lib.load().impeller_msm_n_precompute_curve(curve, window_size, target_window))


def window_count(c: int, curve: int = BN254) -> int:
    """The reference's window count ceil(bits / c) (msm.cuh MsmConfig)."""
    return math.ceil(SCALAR_BITS[curve] / c)


# ------------------------------------------------------ continuous batching

class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("points", ctypes.c_uint64),
                ("peak_bytes", ctypes.c_uint64), ("budget_bytes", ctypes.c_uint64), ("mean_batch", ctypes.c_double),
                ("span_s", ctypes.c_double), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("max_concurrent", ctypes.c_uint64)]


class MsmServer:
    """Continuous-batching MSM server on a context (impeller_server_* C ABI).

    submit() queues a job and returns at once; jobs that arrive while others
    run are admitted as batch slots and HBM free up and run overlapped with
    them; wait() returns the affine result (the context curve's point words)
    and the job's latency."""

    def __init__(self, ctx: MsmContext, max_batch: int = 64, max_inflight: int = 3, hbm_budget: int = 0):
        L = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(L.impeller_server_create(ctypes.byref(h), ctx.handle, max_batch, max_inflight, hbm_budget),
                   "impeller_server_create")
        self.handle = h
        self.ctx = ctx
        self._keep: dict = {}

    def submit(self, h_scalars: np.ndarray) -> int:
        sc = np.ascontiguousarray(h_scalars, dtype=np.uint32).reshape(-1, 8)
        jid = ctypes.c_uint64()
        _lib.check(_lib.load().impeller_server_submit(self.handle, sc.ctypes.data, sc.shape[0], ctypes.byref(jid)),
                   "impeller_server_submit")
        self._keep[jid.value] = sc
        return jid.value

    def submit_raw(self, ptr: int, n: int) -> int:
        """Submit scalars the caller keeps alive (host pointer, n x 8 u32)."""
        jid = ctypes.c_uint64()
        _lib.check(_lib.load().impeller_server_submit(self.handle, ptr, n, ctypes.byref(jid)),
                   "impeller_server_submit")
        return jid.value

    def wait(self, job: int):
        out = np.zeros(self.ctx.pw, dtype=np.uint32)
        lat = ctypes.c_double()
        rc = _lib.load().impeller_server_wait(self.handle, job, out.ctypes.data, ctypes.byref(lat))
        self._keep.pop(job, None)
        _lib.check(rc, "MSM job")
        return out, lat.value

    def poll(self, job: int):
        out = np.zeros(self.ctx.pw, dtype=np.uint32)
        lat = ctypes.c_double()
        rc = _lib.load().impeller_server_poll(self.handle, job, out.ctypes.data, ctypes.byref(lat))
        if rc == 600:  # cudaErrorNotReady
            return None
        self._keep.pop(job, None)
        _lib.check(rc, "MSM job")
        return out, lat.value

    def inject_failures(self, batches: int) -> None:
        _lib.check(_lib.load().impeller_server_inject_failures(self.handle, batches), "inject")

    def stats(self) -> dict:
        st = ServerStats()
        _lib.check(_lib.load().impeller_server_get_stats(self.handle, ctypes.byref(st)), "stats")
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def close(self) -> None:
        if self.handle:
            _lib.load().impeller_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


if __name__ == "__main__":
    # Profiling driver: python -m impeller_b200.msm [bn254|bls12381] [log_n] [table_c] [steps]
    # (device-generated points and scalars, one resident table set for window
    # table_c (0: plain windows), three warm-up MSMs, then `steps` more).
    import sys

    import torch
    curve = {"bn254": BN254, "bls12381": BLS12381}[sys.argv[1] if len(sys.argv) > 1 else "bn254"]
    log_n = int(sys.argv[2]) if len(sys.argv) > 2 else 20
    table_c = int(sys.argv[3]) if len(sys.argv) > 3 else 20
    steps = int(sys.argv[4]) if len(sys.argv) > 4 else 2
    n = 1 << log_n
    ctx = MsmContext(gen_points_device(n, seed=0, curve=curve), curve=curve)
    if table_c:
        ctx.precompute(table_c)
    sc = gen_scalars_device(n, seed=0, stream_id=1, curve=curve)
    for _ in range(3 + steps):
        ctx.msm_device(sc, c=table_c)
    torch.cuda.synchronize()
    ctx.close()
    print(f"{3 + steps} MSMs of 2^{log_n} on {CURVE_NAMES[curve]} done")
