#!/usr/bin/env python
"""BN254 G1 MSM benchmark on B200 (one JSON line on rank 0).

Workload (step): one plain MSM over n = 2^22 affine points P_i = r_i * G
(r_i uniform in Fr, seed 0) with uniform Fr scalars in Montgomery form,
window c from the autotune table.  `value` = points/s with points and scalars
resident in HBM (kernel-only, CUDA events on the launching stream, max over
ranks); `e2e` = the same MSM through the reference-facing C ABI msm() with
pinned host buffers (points and scalars copied in, the 64-byte result copied
out, every step).  N > 1 GPUs run independent replicas (weak scaling).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl impeller|reference]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BN254 MSM points/s at 2^22; batched vs per-call speedup; p50/p99 latency"
UNIT = "points/s"


def workload_name(log2n: int) -> str:
    """The workload both arms time, by the same name."""
    return f"plain single BN254 G1 MSM, n=2^{log2n}, P_i = r_i*G (seed 0), uniform Fr scalars"


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sms, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sms.append(float(parts[0]))
                maxs.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": max(maxs) if maxs else None,
                "reasons": sorted(reasons), "samples": len(sms)}


# ----------------------------------------------------------- algorithmics

def signed_digit_stats(scalars_canonical: np.ndarray, c: int, shared: bool = False,
                       windows: int | None = None) -> tuple[int, int]:
    """(nonzero signed digits, nonempty buckets) of the engine's recoding for
    canonical scalars (n x 8 u32): the entry count of the accumulate phase.
    shared: every digit window uses one bucket set (resident window tables).
    windows: digit windows (BN254 default ceil(254 / c))."""
    s = scalars_canonical.astype(np.uint64)
    words = [s[:, 2 * k] | (s[:, 2 * k + 1] << np.uint64(32)) for k in range(4)]
    W = windows or math.ceil(254 / c)
    half = 1 << (c - 1)
    carry = np.zeros(s.shape[0], dtype=np.int64)
    nonzero, buckets = 0, 0
    used = set()
    for w in range(W):
        o = w * c
        k, sh = divmod(o, 64)
        v = words[k] >> np.uint64(sh)
        if sh + c > 64 and k + 1 < 4:
            v |= words[k + 1] << np.uint64(64 - sh)
        d = (v & np.uint64((1 << c) - 1)).astype(np.int64) + carry
        if w + 1 < W:
            neg = d >= half
            mag = np.where(neg, (1 << c) - d, d)
            carry = neg.astype(np.int64)
        else:
            mag = d
        nz = mag != 0
        nonzero += int(nz.sum())
        if shared:
            used.update(np.unique(mag[nz]).tolist())
        else:
            buckets += int(np.unique(mag[nz]).size)
    return nonzero, (len(used) if shared else buckets)


# DRAM bytes per k_accumulate launch, measured with ncu (dram__bytes_read.sum
# + dram__bytes_write.sum) on the same kernel at n = 2^21 with window tables
# c = 20 (3.607 GB + 0.071 GB) and scaled to n = 2^22 by the number of
# entries (traffic grows in proportion): used when the run matches.
NCU_TRAFFIC_2E22_TABLES_C20 = 7.36e9

# One Fq Montgomery product is 8 rows x (8 products a_j*b_i, 1 for the
# reduction factor, 8 products m*N_j) = 136 32x32->64-bit partial products; a
# Montgomery square takes 36 + 8 + 64 = 108 (symmetric cross products).  A
# mixed XYZZ + affine addition (madd-2008-s) is 8 products and 2 squares:
# 1304 partial products.
PRODUCTS_PER_MUL = 136
PRODUCTS_PER_SQR = 108
MULS_PER_MADD = 10
PRODUCTS_PER_MADD = 8 * PRODUCTS_PER_MUL + 2 * PRODUCTS_PER_SQR


# ------------------------------------------------------------- reference

def reference_gpu(args, n: int, cores: int, pts: np.ndarray, scal: list) -> dict:
    """The reference's own GPU MSM (core/src/msm/src/msm.cu built unmodified
    for sm_100a) on the full n-point workload, driven through its msm() C ABI
    as its Rust operator drives it: pinned host points and scalars, one
    blocking call per MSM (uploads, kernels, host reduction), wall clock.
    Inputs come from the CPU oracle's generators; nothing of this library
    runs here.  Two configurations: MsmConfig::default() and the reference
    cost model's choice for 2^22."""
    try:
        import torch
        from oracle import ref_gpu as RG
    except Exception as e:  # pragma: no cover
        return {"unavailable": f"import failed: {e}"}
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    configs = (("default", RG.DEFAULT_CONFIG, 1), ("cost_model_2e22", RG.TUNED_2E22_CONFIG, RG.TUNED_2E22_PARTS))
    if not all(RG.available(*cfg) for _, cfg, _ in configs):
        return {"unavailable": "reference sm_100a MSM libraries not built (reference sources absent at build time)"}
    from oracle import oracle as O
    out = {"n": n, "api": "reference msm() C ABI (core/src/msm/src/msm.h:4-11), sm_100a build of its sources, "
                          "pinned host buffers, blocking, wall clock", "unit": UNIT}
    for name, (c, alpha), parts in configs:
        ref = RG.RefGpuMsm(pts, c, alpha, parts=parts)
        ms = ref.time_calls(scal, warmup=max(2, args.warmup), steps=args.steps)
        out[name] = {"window_size": c, "target_window": alpha, "parts": parts, "n_precompute": ref.k,
                     "ms_per_call": ms, "value": n / (ms / 1e3)}
        ref.close()
    if RG.available(16, 16, curve=RG.BLS12381):
        # the same call on the reference's second curve (its msm.cu built for bls12381)
        bp = O.gen_points(n, seed=0, threads=cores, curve=O.BLS12381)
        bs = [O.gen_scalars(n, seed=0, stream=1 + v, threads=cores, curve=O.BLS12381) for v in range(2)]
        ref = RG.RefGpuMsm(bp, 16, 16, curve=RG.BLS12381)
        ms = ref.time_calls(bs, warmup=max(2, args.warmup), steps=args.steps)
        out["bls12381_default"] = {"window_size": 16, "target_window": 16, "parts": 1, "ms_per_call": ms,
                                   "value": n / (ms / 1e3)}
        ref.close()
    return out


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU MSM (the C restatement of
    core/tests/msm_halo2.rs best_multiexp; the Rust original cannot be built
    here) on all of the box's host cores, one full 2^22-point MSM per step,
    as the reference's own test times best_multiexp on the whole input
    (core/tests/msm.rs:155-163).  The line also carries `reference_gpu`: the
    reference's own sm_100a MSM kernel on the same workload on the same B200."""
    if rank != 0:
        return
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    n_full = 1 << args.log2n
    pts = O.gen_points(n_full, seed=0, threads=cores)
    scal = [O.gen_scalars(n_full, seed=0, stream=1 + v, threads=cores) for v in range(2)]
    gpu_leg = reference_gpu(args, n_full, cores, pts, scal)
    for w in range(args.warmup):
        O.msm(pts, scal[w % 2], threads=cores)
    t0 = time.perf_counter()
    for k in range(args.steps):
        O.msm(pts, scal[k % 2], threads=cores)
    dt = (time.perf_counter() - t0) / args.steps
    value = n_full / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (254-bit Montgomery)", "data": "synthetic (seeded r_i*G, uniform Fr)",
        "config": {"workload": workload_name(args.log2n), "n": n_full, "threads": cores,
                   "cpu": "the whole input per step, all host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"the full 2^{args.log2n}-point MSM per step (two alternating scalar vectors)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": gpu_leg,
        "reference_gpu_ntt": reference_gpu_ntt(args),
    }
    print(json.dumps(line), flush=True)


def reference_gpu_ntt(args, log_n: int = 24) -> dict:
    """The reference's own NTT kernels (core/src/ntt/src/ntt.cu built
    unmodified for sm_100a, NTT_FIELD=bn254_fr) on 2^24 device-resident
    BN254 Fr elements with the launch shape its operator uses ((8, 8),
    core/src/ntt.rs:383-388), CUDA events.  Inputs and twiddles come from
    the CPU oracle; nothing of this library runs here."""
    try:
        import ctypes as C
        import torch
        from oracle import oracle as O
    except Exception as e:  # pragma: no cover
        return {"unavailable": f"import failed: {e}"}
    path = os.path.join(ROOT, "oracle", "_ref", "libref_ntt_bn254_fr.so")
    if not torch.cuda.is_available() or not os.path.exists(path):
        return {"unavailable": "no CUDA device or reference NTT library not built"}

    class PolyPtr(C.Structure):
        _fields_ = [("ptr", C.c_void_p), ("len", C.c_size_t), ("rotate", C.c_size_t), ("offset", C.c_size_t),
                    ("whole_len", C.c_size_t)]

    ref = C.CDLL(path)
    ref.ssip_ntt.restype = C.c_int
    ref.ssip_ntt.argtypes = [PolyPtr, C.c_void_p, C.c_uint, C.c_void_p, C.c_uint, C.c_uint]
    ref.recompute_ntt.restype = C.c_int
    ref.recompute_ntt.argtypes = [PolyPtr, C.c_void_p, C.c_uint, C.c_void_p, C.c_uint, C.c_void_p, C.c_uint,
                                  C.c_uint]
    n = 1 << log_n
    cores = os.cpu_count() or 1
    x = torch.from_numpy(O.gen_scalars(n, seed=7, stream=11, threads=cores).view(np.int32)).cuda()
    u = O.mont_limbs(O.root_of_unity(log_n))
    tw = torch.from_numpy(O.ntt_roots(n // 2, u).view(np.int32)).cuda()
    # pq_deg as the reference's GenPqOmegas::get_pq_len gives it for (8, 8) launch shapes
    # (core/src/ntt.rs:340-355): max(deg_stage1, deg_stage2)
    def get_deg(d, m):
        r = 1
        while True:
            x = d if r == 1 else (d - 1) // r + 1
            if x <= m:
                return x
            r += 1
    deg = max(get_deg((log_n + 1) // 2, 9), get_deg(log_n // 2, 5))
    pq, om = O.pq_omegas(deg, n, u)
    d_pq = torch.from_numpy(pq.view(np.int32)).cuda()
    d_om = torch.from_numpy(om.view(np.int32)).cuda()
    stream = torch.cuda.current_stream()
    p = PolyPtr(x.data_ptr(), n, 0, 0, n)

    def timed(call):
        for _ in range(max(3, args.warmup)):
            if call() != 0:
                raise RuntimeError("reference NTT call failed")
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    st = stream.cuda_stream
    ms = timed(lambda: ref.ssip_ntt(p, tw.data_ptr(), log_n, st, 8, 8))
    ms_re = timed(lambda: ref.recompute_ntt(p, d_pq.data_ptr(), deg, d_om.data_ptr(), log_n, st, 8, 8))
    return {"workload": f"in-place forward NTT, BN254 Fr, n=2^{log_n}", "n": n, "unit": "elements/s",
            "ssip_ntt": {"ms_per_step": ms, "value": n / (ms * 1e-3)},
            "recompute_ntt": {"ms_per_step": ms_re, "value": n / (ms_re * 1e-3)},
            "api": "reference ssip_ntt / recompute_ntt C ABI (core/src/ntt/src/ntt.h), CUDA events"}


# ------------------------------------------------------------------ main

def max_over_ranks(ms: float, dist=None, device=None) -> float:
    """The slowest rank's time (every rank runs the same collective)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(n_per_rank: int, world: int, ms_max: float) -> float:
    """Weak scaling: every rank runs its own n-point MSM; whole-job points/s."""
    return world * n_per_rank / (ms_max / 1e3)


def cpu_baseline(pts_host: np.ndarray, scal_host: np.ndarray) -> dict:
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    m = 1 << 16
    t0 = time.perf_counter()
    O.msm(pts_host[:m], scal_host[:m], threads=cores)
    dt = time.perf_counter() - t0
    # grow the sample to about 10 s of CPU work (at most 2^20 points)
    while m < min(pts_host.shape[0], 1 << 20) and dt * 2.2 < 10.0:
        m *= 2
        t0 = time.perf_counter()
        O.msm(pts_host[:m], scal_host[:m], threads=cores)
        dt = time.perf_counter() - t0
    return {"value": m / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"first 2^{int(math.log2(m))} points/scalars of the workload, one MSM, {dt:.2f} s"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="impeller", choices=["impeller", "reference"])
    ap.add_argument("--log2n", type=int, default=22)
    ap.add_argument("--no-extras", action="store_true", help="skip e2e / batched / CPU legs")
    ap.add_argument("--only", default="", help="comma list of extra legs to run (e2e, resident, batched, served, cpu, "
                                               "bls12381, ntt); default all")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", args.gpus if args.gpus else 1)
    local = env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from impeller_b200 import msm as M
    from impeller_b200 import lib as L
    lib = L.load()
    n = 1 << args.log2n
    dev = local
    stream = torch.cuda.current_stream()

    srs_log2 = max(args.log2n, 23 if not args.no_extras else args.log2n)
    pts = M.gen_points_device(1 << srs_log2, seed=0, device=dev)  # SRS; the MSM uses its first n points
    V = 4  # rotating scalar vectors: 4 x 128 MiB + 256 MiB of points, inputs > L2
    scal = [M.gen_scalars_device(n, seed=0, stream_id=1 + v, device=dev) for v in range(V)]
    ctx = M.MsmContext(pts, device=dev)
    c_tab = M.table_window(n)  # resident window tables where the autotune table says they win
    t0 = time.perf_counter()
    if c_tab:
        ctx.precompute(c_tab)
    precompute_s = time.perf_counter() - t0
    c = ctx.window(n)
    outs = [torch.empty(16, dtype=torch.int32, device=f"cuda:{dev}") for _ in range(V)]

    def barrier():
        if dist is not None:
            dist.barrier()

    for w in range(args.warmup):
        ctx.msm_device(scal[w % V], c=c, out=outs[w % V])
    torch.cuda.synchronize()

    lib.impeller_ctx_profile(ctx.handle, 1)
    sampler = ClockSampler(dev)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        ctx.msm_device(scal[k % V], c=c, out=outs[k % V])
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    ms_max = max_over_ranks(ms, dist, device=f"cuda:{dev}")
    value = replica_value(n, world, ms_max)

    phases = (ctypes.c_double * 8)()
    runs = ctypes.c_uint32()
    L.check(lib.impeller_ctx_profile_read(ctx.handle, phases, 8, ctypes.byref(runs)))
    lib.impeller_ctx_profile(ctx.handle, 0)
    nr = max(1, runs.value)
    phase_ms = {lib.impeller_phase_name(i).decode(): phases[i] / nr for i in range(8)}

    line = None
    if rank == 0:
        # algorithmic work of the dominant kernel (accumulate) on the timed inputs
        canon = [M.to_host(M.gen_scalars_device(n, seed=0, stream_id=1 + v, mont=False, device=dev)).reshape(n, 8)
                 for v in range(V)]
        stats = [signed_digit_stats(cv, c, shared=bool(c_tab)) for cv in canon]
        madds = statistics.mean(nz - nb for nz, nb in stats)
        entries = statistics.mean(nz for nz, _ in stats)
        peak = ctypes.c_double()
        L.check(lib.impeller_imad_peak(dev, ctypes.byref(peak)))
        acc_ms = phase_ms["accumulate"]
        achieved = madds * PRODUCTS_PER_MADD / (acc_ms * 1e-3) / 1e9
        hbm_peak = None
        try:
            hbm_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        except Exception:
            hbm_peak = 6650.0
        sort_ms = phase_ms["histogram"] + phase_ms["scan"] + phase_ms["scatter"]
        nbk = (1 << (c - 1)) * (1 if c_tab else math.ceil(254 / c))
        sort_bytes = 2 * 32 * n + 4 * entries + 3 * 4 * nbk
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 (254-bit Montgomery, 8x32-bit limbs)",
            "data": "synthetic: P_i = r_i*G (r_i uniform Fr, seed 0), uniform Fr scalars (seeded streams)",
            "config": {"workload": workload_name(args.log2n), "n": n, "window": c, "window_source": "autotune table",
                       "window_tables": bool(c_tab),
                       "window_tables_setup_s": round(precompute_s, 3) if c_tab else None,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs > L2: 256 MiB points + 4 rotating 128 MiB scalar vectors"},
            "gpu_launches": args.steps * ctx.launches(n, c),
            "phase_ms": {k: round(v, 4) for k, v in phase_ms.items()},
            "roofline": {"bound": "imad", "kernel": "k_accumulate", "achieved": achieved, "peak": peak.value,
                         "unit": "G 32x32->64 products/s", "frac": achieved / peak.value,
                         "traffic": NCU_TRAFFIC_2E22_TABLES_C20 if (args.log2n == 22 and c_tab == 20 and c == 20)
                         else None,
                         "algorithmic_bytes": madds * (64 + 4),
                         "per_launch": {"madds": madds, "products_per_madd": PRODUCTS_PER_MADD,
                                        "madds_per_s": madds / (acc_ms * 1e-3), "ms": acc_ms},
                         "peak_source": "impeller_imad_peak: independent Fq Montgomery products (4 chains/thread, 136 partial products each), measured live"},
            "clocks": clocks,
        }
        # the decompose + sort phase, bound by HBM: reported inside `roofline`
        # so that it stays beside the headline kernel's figures
        line["roofline"]["sort"] = {
            "bound": "hbm", "kernels": "sort phase (every kernel from the scalar read to the bucket-ordered entries)",
            "ms": sort_ms, "algorithmic_bytes": sort_bytes, "achieved": sort_bytes / (sort_ms * 1e-3) / 1e9,
            "peak": hbm_peak, "unit": "GB/s", "frac": sort_bytes / (sort_ms * 1e-3) / 1e9 / hbm_peak,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}

    legs = set(args.only.split(",")) if args.only else {"e2e", "resident", "batched", "served", "cpu", "bls12381",
                                                         "ntt"}
    if not args.no_extras and rank == 0:
        if "e2e" in legs:
            line["e2e"] = e2e_reference_abi(M, pts[:n], scal[0], n, c, args)
        if "resident" in legs:
            line["e2e_resident_srs"] = e2e_resident(M, ctx, scal[0], n, c, args)
        if "batched" in legs:
            line["batched"] = batched_vs_per_call(M, ctx, dev, args)
        if "served" in legs:
            line["served"] = served_stream(M, ctx, dev, args)
        if "cpu" in legs:
            pts_host = M.to_host(pts[: 1 << 20]).reshape(-1, 16)
            sc_host = M.to_host(scal[0][: 1 << 20]).reshape(-1, 8)
            line["cpu_baseline"] = cpu_baseline(pts_host, sc_host)
    if not args.no_extras and rank == 0 and "bls12381" in legs:
        del scal
        ctx.close()
        del pts
        torch.cuda.empty_cache()
        line["bls12381"] = bls12381_leg(M, dev, n, args, peak.value)
    if not args.no_extras and rank == 0 and "ntt" in legs:
        torch.cuda.empty_cache()
        line["ntt"] = ntt_leg(M, dev, args, peak.value)
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def e2e_reference_abi(M, d_pts, d_scal, n, c, args) -> dict:
    """The reference's calling convention: host points and scalars (pinned),
    blocking msm() that uploads both, computes and returns the affine point."""
    import torch
    c = M.default_window(n)  # the drop-in path has no resident tables: best plain window
    cfg = M.MsmConfig(window_size=c, target_window=math.ceil(254 / c))
    op = M.MSM(cfg)
    buf, keep = M.alloc_gpu_buffer(op.get_buffer_size(n)[0])
    hp = torch.empty((n, 16), dtype=torch.int32, pin_memory=True)
    hs = torch.empty((n, 8), dtype=torch.int32, pin_memory=True)
    hp.copy_(d_pts.cpu())
    hs.copy_(d_scal.cpu())
    pts_np = hp.numpy().view(np.uint32)
    sc_np = hs.numpy().view(np.uint32)
    torch.cuda.synchronize()
    for _ in range(2):
        op.run([pts_np], [sc_np], [buf])
    steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(steps):
        op.run([pts_np], [sc_np], [buf])
    dt = (time.perf_counter() - t0) / steps
    del keep
    return {"value": n / dt, "unit": UNIT, "h2d_bytes_per_step": n * (64 + 32), "d2h_bytes_per_step": 64,
            "ms_per_step": dt * 1e3, "api": f"msm() C ABI ({M.lib_name(cfg)}), pinned host buffers, wall clock"}


def ntt_leg(M, dev, args, imad_peak: float, log_n: int = 24) -> dict:
    """The NTT operator (the reference's ssip_ntt / recompute_ntt, BN254 Fr):
    one in-place forward transform of 2^24 device-resident elements per step,
    CUDA events on the launching stream (512 MiB of data, > L2); the same
    through host buffers (pinned polynomial uploaded and read back every
    step); the recompute variant.  Roofline: Montgomery products per second
    against the live integer-multiply ceiling, and HBM bytes moved."""
    import torch
    from impeller_b200 import ntt as NT
    n = 1 << log_n
    x = M.gen_scalars_device(n, seed=7, stream_id=11, device=dev)
    w = NT.root_of_unity(log_n)
    tw_h = np.zeros((n // 2, 8), np.uint32)
    t0 = time.perf_counter()
    NT.SsipPrecompute().get_fn()(tw_h, NT.to_mont_limbs(w))
    precompute_s = time.perf_counter() - t0
    tw = torch.from_numpy(tw_h.view(np.int32)).to(f"cuda:{dev}")
    f = NT.SsipNtt().get_fn()
    stream = torch.cuda.current_stream()

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms = timed(lambda: f(x, tw), args.steps)
    g = NT.GenPqOmegas()
    pq = np.zeros((g.get_pq_len(log_n), 8), np.uint32)
    om = np.zeros((32, 8), np.uint32)
    g.get_fn()(pq, om, n, NT.to_mont_limbs(w))
    d_pq = torch.from_numpy(pq.view(np.int32)).to(f"cuda:{dev}")
    d_om = torch.from_numpy(om.view(np.int32)).to(f"cuda:{dev}")
    fr = NT.RecomputeNtt().get_fn()
    ms_re = timed(lambda: fr(x, d_pq, d_om), args.steps)
    # host buffers: upload, transform, read back
    hx = torch.empty((n, 8), dtype=torch.int32, pin_memory=True)
    hx.copy_(x.cpu())
    ho = torch.empty((n, 8), dtype=torch.int32, pin_memory=True)

    def e2e_step():
        x.copy_(hx, non_blocking=True)
        f(x, tw)
        ho.copy_(x, non_blocking=True)

    ms_e2e = timed(e2e_step, max(3, args.steps // 2))
    prods = NT.butterfly_products(log_n) * PRODUCTS_PER_MUL
    passes = NT.launches(log_n)
    hbm_bytes = passes * 2 * 32 * n + 32 * n  # every pass reads and writes the data; twiddles about one more read
    achieved = prods / (ms * 1e-3) / 1e9
    return {"workload": f"in-place forward NTT, BN254 Fr, n=2^{log_n}, natural order", "n": n,
            "value": n / (ms * 1e-3), "unit": "elements/s", "ms_per_step": ms,
            "gpu_launches_per_step": passes, "twiddle_precompute_s": round(precompute_s, 3),
            "recompute": {"ms_per_step": ms_re, "value": n / (ms_re * 1e-3)},
            "e2e": {"value": n / (ms_e2e * 1e-3), "unit": "elements/s", "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": 32 * n, "d2h_bytes_per_step": 32 * n,
                    "api": "ssip_ntt C ABI between pinned-host copies, CUDA events"},
            "roofline": {"bound": "imad", "kernel": "k_ntt_pass", "achieved": achieved, "peak": imad_peak,
                         "unit": "G 32x32->64 products/s", "frac": achieved / imad_peak,
                         "products_per_step": prods,
                         "hbm_gbs_achieved": hbm_bytes / (ms * 1e-3) / 1e9,
                         "peak_source": "impeller_imad_peak, measured live"}}


def bls12381_leg(M, dev, n, args, imad_peak: float) -> dict:
    """The same MSM on the reference's second curve, BLS12-381 G1 (381-bit
    base field in 12 limbs, 255-bit scalars): device-resident inputs timed
    with CUDA events (resident window tables where the autotune table puts
    them), then the drop-in msm() C ABI of lib/libmsm_bls12381_{c}_{alpha}
    on pinned host buffers, wall clock."""
    import torch
    C = M.BLS12381
    pts = M.gen_points_device(n, seed=0, device=dev, curve=C)
    scal = [M.gen_scalars_device(n, seed=0, stream_id=1 + v, device=dev, curve=C) for v in range(4)]
    ctx = M.MsmContext(pts, device=dev, curve=C)
    c_tab = M.table_window(n)
    if c_tab:
        ctx.precompute(c_tab)
    c = ctx.window(n)
    outs = [torch.empty(24, dtype=torch.int32, device=f"cuda:{dev}") for _ in range(4)]
    stream = torch.cuda.current_stream()
    from impeller_b200 import lib as L
    lib = L.load()
    for w in range(args.warmup):
        ctx.msm_device(scal[w % 4], c=c, out=outs[w % 4])
    torch.cuda.synchronize()
    lib.impeller_ctx_profile(ctx.handle, 1)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        ctx.msm_device(scal[k % 4], c=c, out=outs[k % 4])
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    phases = (ctypes.c_double * 8)()
    runs = ctypes.c_uint32()
    L.check(lib.impeller_ctx_profile_read(ctx.handle, phases, 8, ctypes.byref(runs)))
    nr = max(1, runs.value)
    phase_ms = {lib.impeller_phase_name(i).decode(): phases[i] / nr for i in range(8)}
    ctx.close()
    # accumulate-phase roofline: 12-limb Montgomery products (12 rows of
    # 12 + 1 + 12 partial products = 300) x 10 per mixed addition
    W = math.ceil(255 / c) + (1 if c in (3, 5, 15, 17) else 0)
    stats = [signed_digit_stats(M.to_host(M.gen_scalars_device(n, seed=0, stream_id=1 + v, mont=False, device=dev,
                                                                curve=C)).reshape(n, 8), c, shared=bool(c_tab),
                                windows=W) for v in range(4)]
    madds = statistics.mean(nz - nb for nz, nb in stats)
    acc_ms = phase_ms["accumulate"]
    achieved = madds * MULS_PER_MADD * 300 / (acc_ms * 1e-3) / 1e9
    bls_peak = ctypes.c_double()
    L.check(lib.impeller_imad_peak_curve(dev, C, ctypes.byref(bls_peak)))
    # drop-in ABI, host buffers
    cd = M.default_window(n, C)
    cfg = M.MsmConfig(window_size=cd, target_window=M.window_count(cd, C), curve=C)
    op = M.MSM(cfg)
    buf, keep = M.alloc_gpu_buffer(op.get_buffer_size(n)[0], device=dev)
    hp = torch.empty((n, 24), dtype=torch.int32, pin_memory=True)
    hs = torch.empty((n, 8), dtype=torch.int32, pin_memory=True)
    hp.copy_(pts.cpu())
    hs.copy_(scal[0].cpu())
    del pts, scal
    pts_np, sc_np = hp.numpy().view(np.uint32), hs.numpy().view(np.uint32)
    for _ in range(2):
        op.run([pts_np], [sc_np], [buf])
    steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(steps):
        op.run([pts_np], [sc_np], [buf])
    dt = (time.perf_counter() - t0) / steps
    del keep
    return {"workload": f"single BLS12-381 G1 MSM, n=2^{int(math.log2(n))}, window c={c}",
            "window_tables": bool(c_tab), "value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "phase_ms": {k: round(v, 4) for k, v in phase_ms.items()},
            "roofline": {"bound": "imad", "kernel": "k_accumulate<Bls12381>", "achieved": achieved,
                         "peak": bls_peak.value, "unit": "G 32x32->64 products/s",
                         "frac": achieved / bls_peak.value,
                         "per_launch": {"madds": madds, "products_per_madd": MULS_PER_MADD * 300, "ms": acc_ms},
                         "peak_8limb": imad_peak,
                         "peak_source": "impeller_imad_peak_curve: independent 12-limb BLS12-381 Fq products "
                                        "(4 chains/thread, 300 partial products each), measured live"},
            "timing": "CUDA events, inputs resident, 4 rotating scalar vectors (> L2)",
            "e2e": {"value": n / dt, "unit": UNIT, "h2d_bytes_per_step": n * (96 + 32), "d2h_bytes_per_step": 96,
                    "ms_per_step": dt * 1e3, "api": f"msm() C ABI ({M.lib_name(cfg)}), pinned host buffers, "
                                                    "wall clock"}}


def e2e_resident(M, ctx, d_scal, n, c, args) -> dict:
    import torch
    hs = torch.empty((n, 8), dtype=torch.int32, pin_memory=True)
    hs.copy_(d_scal.cpu())
    sc_np = hs.numpy().view(np.uint32)
    for _ in range(2):
        ctx.msm_host(sc_np, c=c)
    steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.msm_host(sc_np, c=c)
    dt = (time.perf_counter() - t0) / steps
    return {"value": n / dt, "unit": UNIT, "h2d_bytes_per_step": n * 32, "d2h_bytes_per_step": 64,
            "ms_per_step": dt * 1e3, "api": "impeller_msm_host (points resident), pinned scalars, wall clock"}


def served_stream(M, ctx, dev, args, seconds: float = 6.0, rate: float = 200.0) -> dict:
    """Poisson arrivals (mean 200 jobs/s) of MSM jobs with sizes log-uniform in
    [2^12, 2^23] over the resident 2^23-point SRS, served with continuous
    batching; every job's scalars are a slice of one pinned host buffer."""
    import torch
    nmax = 1 << 23
    for ct in sorted({M.table_window(1 << k) for k in range(12, 24)} - {0}):
        ctx.precompute(ct)
    host = torch.empty((nmax, 8), dtype=torch.int32, pin_memory=True)
    host.copy_(M.gen_scalars_device(nmax, seed=0, stream_id=77, device=dev).cpu())
    base = host.data_ptr()
    rng = np.random.default_rng(0)
    jobs = []
    t = 0.0
    while t < seconds:
        t += rng.exponential(1.0 / rate)
        n = int(round(2 ** rng.uniform(12, 23)))
        off = int(rng.integers(0, nmax - n + 1))
        jobs.append((t, n, off))
    # up to 16 batches in flight (the server's limit): each arriving job
    # starts at once on a free stream; with 3, p99 was 74-90 ms, with 12-16
    # about 60 ms, at the same throughput (the offered load)
    srv = M.MsmServer(ctx, max_batch=64, max_inflight=16)
    ids = []
    t0 = time.perf_counter()
    for (ta, n, off) in jobs:
        delay = ta - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit_raw(base + off * 32, n))
    results = [srv.wait(j)[0] for j in ids]
    st = srv.stats()
    srv.close()
    # bit-exactness in the mix: a sample of jobs again, alone
    checks = rng.choice(len(jobs), size=min(12, len(jobs)), replace=False)
    same = all(np.array_equal(results[i], ctx.msm_host(host[jobs[i][2]: jobs[i][2] + jobs[i][1]].numpy()
                                                          .view(np.uint32))) for i in checks)
    total = sum(n for _, n, _ in jobs)
    return {"workload": f"Poisson {rate:g} jobs/s for {seconds:g} s, n log-uniform in [2^12, 2^23], 2^23 SRS",
            "jobs": len(jobs), "points": total, "points_per_s": total / st["span_s"] if st["span_s"] else None,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"], "mean_ms": st["mean_ms"],
            "batches": st["batches"], "mean_batch": st["mean_batch"], "max_concurrent": st["max_concurrent"],
            "peak_hbm_bytes": st["peak_bytes"], "sample_same_alone_and_in_mix": bool(same),
            "sample_checked": int(len(checks))}


def batched_vs_per_call(M, ctx, dev, args) -> dict:
    """64 MSMs, sizes log-uniform in [2^10, 2^20] (seed 0), over prefixes of
    the resident SRS: one batched CUDA-graph run vs 64 per-call MSMs."""
    import torch
    rng = np.random.default_rng(0)
    sizes = [int(round(2 ** rng.uniform(10, 20))) for _ in range(64)]
    for ct in sorted({M.table_window(s) for s in sizes} - {0}):
        ctx.precompute(ct)  # every table set the batch's sizes use (resident next to the SRS)
    scal = [M.gen_scalars_device(s, seed=0, stream_id=1000 + i, device=dev) for i, s in enumerate(sizes)]
    total = sum(sizes)
    b = ctx.batch(sizes, graph=True)
    out = torch.empty((64, 16), dtype=torch.int32, device=f"cuda:{dev}")
    outs = [torch.empty(16, dtype=torch.int32, device=f"cuda:{dev}") for _ in sizes]
    st = torch.cuda.current_stream()
    for _ in range(3):
        b.run(scal, out=out)
        for i, s in enumerate(sizes):
            ctx.msm_device(scal[i], n=s, out=outs[i])
    torch.cuda.synchronize()
    reps = 5
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record(st)
    for _ in range(reps):
        b.run(scal, out=out)
    e[1].record(st)
    for _ in range(reps):
        for i, s in enumerate(sizes):
            ctx.msm_device(scal[i], n=s, out=outs[i])
    e[2].record(st)
    torch.cuda.synchronize()
    tb = e[0].elapsed_time(e[1]) / reps
    tp = e[1].elapsed_time(e[2]) / reps
    same = bool(torch.equal(out, torch.stack(outs)))
    launches = b.launches
    per_call_launches = sum(ctx.launches(s) for s in sizes)
    b.close()
    # the same plan launched kernel by kernel from the host, without the graph:
    # how much of the batched time the graph's launch savings account for
    b2 = ctx.batch(sizes, graph=False)
    out2 = torch.empty_like(out)
    for _ in range(2):
        b2.run(scal, out=out2)
    torch.cuda.synchronize()
    e[2].record(st)
    for _ in range(reps):
        b2.run(scal, out=out2)
    e[3].record(st)
    torch.cuda.synchronize()
    tng = e[2].elapsed_time(e[3]) / reps
    same = same and bool(torch.equal(out2, out))
    b2.close()
    return {"workload": "64 MSMs, n log-uniform in [2^10, 2^20] (seed 0), prefixes of one resident SRS",
            "total_points": total, "batched_ms": tb, "per_call_ms": tp,
            "batched_points_per_s": total / (tb * 1e-3), "per_call_points_per_s": total / (tp * 1e-3),
            "speedup": tp / tb, "results_identical": same, "launches_per_batch": launches,
            "launches_per_call_total": per_call_launches, "batched_no_graph_ms": tng,
            "graph_saving_ms": tng - tb}


if __name__ == "__main__":
    main()
