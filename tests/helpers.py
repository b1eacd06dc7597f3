"""Shared helpers for the tests (hex fixtures, device plumbing)."""
from __future__ import annotations

import json
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rows(hexrows, width):
    return np.array([[int(r[8 * i:8 * i + 8], 16) for i in range(width)] for r in hexrows],
                    dtype=np.uint32).reshape(-1, width)


def golden_cases():
    data = json.load(open(os.path.join(GOLD, "msm_golden.json")))
    out = []
    for c in data["cases"]:
        out.append((c["name"], rows(c["points"], 16), rows(c["scalars"], 8), rows([c["result"]], 16)[0]))
    return out


def kat():
    return json.load(open(os.path.join(GOLD, "kat.json")))


def h2l(words):
    return np.array([int(w, 16) for w in words], dtype=np.uint32)


def random_field(rng, n, modulus):
    return np.stack([np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(8)], dtype=np.uint32)
                     for x in (int.from_bytes(rng.bytes(32), "little") % modulus for _ in range(n))])


def cuda_ok() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
