"""Window-size autotuner for the B200 MSM.

Measures, on the GPU at hand, the time of one MSM of n = 2^k points for every
candidate window c, both plain (one bucket set per digit window) and with
resident window tables (one shared bucket set, tables 2^(j*c) * P kept in
HBM), and stores the best choice per size as a table:

    impeller_b200/autotune_table.json
    {"device": ..., "entries": [{"log2n": k, "plain_c": c, "plain_ms": t,
                                 "tables_c": c2, "tables_ms": t2}, ...]}

tables_c is 0 when tables do not beat the plain path at that size.  The build
compiles the stored table into libimpeller_msm.so as its default
(csrc/autotune_default.inc, generated by impeller_b200.build), and
load_table() installs a table at run time through impeller_set_window_table.
The reference picks its configuration with a fitted A100 cost model in a
Python subprocess per MSM node (core/src/msm/tuning/cost_model.py,
core/src/msm.rs:36-99); this replaces the model with measurements.

    python -m impeller_b200.autotune [--min 10] [--max 23] [--reps 5]
"""
from __future__ import annotations

import argparse
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE_PATH = os.path.join(HERE, "autotune_table.json")

# window tables: c >= 16 for n >= 2^14, where their top digit window keeps
# >= 12 bits so the shared bucket set is not flooded by the short top window;
# small c for small n, where the flooding is bounded by n and a single shared
# bucket set saves the plain path's Horner tail (about 250 doublings).
TABLE_WINDOWS = (16, 18, 20, 22)
SMALL_TABLE_WINDOWS = (8, 10, 12, 13)
SMALL_TABLE_MAX_LOG2N = 17


def plain_candidates(k: int) -> list:
    centre = max(5, min(20, int(round(0.75 * k))))
    return sorted({c for c in range(centre - 3, centre + 3) if 4 <= c <= 22})


def _time(ctx, scal, n, c, reps) -> float:
    import torch
    out = torch.empty(16, dtype=torch.int32, device=f"cuda:{ctx.device}")
    ctx.msm_device(scal, n=n, c=c, out=out)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        ctx.msm_device(scal, n=n, c=c, out=out)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune(kmin: int = 10, kmax: int = 23, reps: int = 5, device: int = 0, out: str = TABLE_PATH) -> dict:
    import torch

    from . import msm as M
    torch.cuda.set_device(device)
    nmax = 1 << kmax
    pts = M.gen_points_device(nmax, seed=0, device=device)
    scal = M.gen_scalars_device(nmax, seed=0, stream_id=7, device=device)
    ctx = M.MsmContext(pts, device=device)
    entries = {k: {"log2n": k} for k in range(kmin, kmax + 1)}
    for k in range(kmin, kmax + 1):
        n = 1 << k
        r = max(2, reps if k < 20 else reps // 2)
        best = min((_time(ctx, scal, n, c, r), c) for c in plain_candidates(k))
        entries[k].update(plain_c=best[1], plain_ms=round(best[0], 4))
        print(json.dumps(entries[k]), flush=True)
    tab = {k: (math.inf, 0) for k in entries}
    for ct in SMALL_TABLE_WINDOWS + TABLE_WINDOWS:
        ctx.precompute(ct)
        ks = range(kmin, min(kmax, SMALL_TABLE_MAX_LOG2N) + 1) if ct in SMALL_TABLE_WINDOWS \
            else range(max(kmin, 14), kmax + 1)
        for k in ks:
            n = 1 << k
            t = _time(ctx, scal, n, ct, max(2, reps // 2))
            if t < tab[k][0]:
                tab[k] = (t, ct)
        print(json.dumps({"tables_c": ct, "ms": {k: round(tab[k][0], 3) for k in tab if tab[k][1] == ct}}),
              flush=True)
    for k, (t, ct) in tab.items():
        good = ct and t < entries[k]["plain_ms"]
        entries[k].update(tables_c=ct if good else 0, tables_ms=round(t, 4) if ct else None)
    ctx.close()
    table = {"device": torch.cuda.get_device_name(device), "reps": reps,
             "entries": [entries[k] for k in sorted(entries)]}
    with open(out, "w") as f:
        json.dump(table, f, indent=1)
    return table


def read_table(path: str = TABLE_PATH) -> dict | None:
    if not os.path.exists(path):
        return None
    return json.load(open(path))


def load_table(path: str = TABLE_PATH) -> bool:
    """Install the stored table in the loaded library (run time)."""
    import ctypes

    from . import lib as L
    t = read_table(path)
    if not t:
        return False
    es = t["entries"]
    cnt = len(es)
    lg = (ctypes.c_uint32 * cnt)(*[e["log2n"] for e in es])
    cp = (ctypes.c_uint32 * cnt)(*[e["plain_c"] for e in es])
    ct = (ctypes.c_uint32 * cnt)(*[e.get("tables_c", 0) or 0 for e in es])
    L.check(L.load().impeller_set_window_table(lg, cp, ct, cnt), "impeller_set_window_table")
    return True


def c_include(path: str = TABLE_PATH) -> str:
    """The compiled-in default table (csrc/autotune_default.inc)."""
    t = read_table(path)
    lines = ["// Generated by impeller_b200/build.py from impeller_b200/autotune_table.json",
             "// (measured by impeller_b200/autotune.py); do not edit.  {log2 n, plain c, tables c}"]
    if t:
        lines.append(f"// device: {t.get('device', '?')}")
        for e in t["entries"]:
            lines.append(f"{{{e['log2n']}u, {e['plain_c']}u, {e.get('tables_c', 0) or 0}u}},")
    return "\n".join(lines) + "\n"


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--min", type=int, default=10)
    ap.add_argument("--max", type=int, default=23)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--out", default=TABLE_PATH)
    a = ap.parse_args()
    tune(a.min, a.max, a.reps, out=a.out)
