"""Generate the golden fixtures under tests/golden/ (run where the reference
sources are mounted; the outputs are committed and the GPU box never needs
the reference).

  python tests/golden/make_golden.py [REF_ROOT]

REF_ROOT defaults to the REF_ROOT environment variable, else to a checkout
named ``reference`` beside this repository.

1. ``kat.json``: the reference's own known-answer vectors, parsed from its
   test sources (all values little-endian u32 limbs, as BIG_INTEGER_CHUNKS8
   stores them):
     - curve:  core/src/common/curve/tests/bn254.cu:174-203
               p1, p2, p1+p2 (pr), p1+100*p2 (pr100), 128*p1 (p1r128);
               Montgomery affine coordinates.
     - Fr:     core/src/common/mont/tests/main.cu instance1 (:238-252),
               instance2 (:369-383), instance3 (:527-532).
2. ``msm_golden.json``: MSM inputs and outputs where the output is computed
   with the reference's OWN host arithmetic (``oracle/_ref/libref_bn254.so``
   wraps core/src/common/curve/src/curve_xyzz.cuh and
   core/src/common/mont/src/field.cuh; double-and-add per term), on seeded
   inputs and on the edge cases the reference's design has to survive
   (zero scalars, identity points, P and -P, repeated points, scalar r-1,
   the skewed witness-like mix).
3. ``generators.json``: the first values of the seeded synthetic streams, so
   that any change to the input definitions is caught.
4. ``msm_golden_bls12381.json`` / ``generators_bls12381.json``: the same for
   the reference's second curve, BLS12-381 G1 (outputs from the reference's
   host arithmetic, core/src/common/curve/src/bls12381.cuh over
   core/src/common/mont/src/bls12381_fq.cuh / bls12381_fr.cuh).  The
   reference ships no BLS12-381 known-answer vectors of its own.
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

CHUNKS = re.compile(
    r"const\s+u32\s+(\w+)\[[^\]]*\]\s*=\s*BIG_INTEGER_CHUNKS(8|16)\(([^)]*)\)")


def parse_chunks(text: str) -> dict[str, list[int]]:
    """name -> little-endian u32 limbs (BIG_INTEGER_CHUNKS lists the most
    significant word first)."""
    out = {}
    for name, _, body in CHUNKS.findall(text):
        words = [int(w.strip(), 16) for w in body.split(",")]
        out.setdefault(name, []).append(list(reversed(words)))
    return out


def parse_namespaces(text: str) -> dict[str, dict[str, list[int]]]:
    res = {}
    for m in re.finditer(r"namespace\s+(instance\d)\s*\{", text):
        start = m.end()
        depth, i = 1, start
        while depth and i < len(text):
            depth += {"{": 1, "}": -1}.get(text[i], 0)
            i += 1
        body = text[start:i]
        res[m.group(1)] = {k: v[0] for k, v in parse_chunks(body).items()}
    return res


def hexlimbs(a) -> list[str]:
    return ["%08x" % int(v) for v in np.asarray(a, dtype=np.uint32).reshape(-1)]


def rows_hex(a) -> list[str]:
    a = np.asarray(a, dtype=np.uint32)
    return ["".join("%08x" % int(v) for v in row) for row in a.reshape(a.shape[0], -1)]


def main(ref_root: str) -> None:
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    if not O.ref_available():
        raise SystemExit("reference harness oracle/_ref/libref_bn254.so not built")

    curve_src = open(os.path.join(ref_root, "core/src/common/curve/tests/bn254.cu")).read()
    mont_src = open(os.path.join(ref_root, "core/src/common/mont/tests/main.cu")).read()
    curve = {k: v[0] for k, v in parse_chunks(curve_src).items()}
    kat = {
        "source": {
            "curve": "core/src/common/curve/tests/bn254.cu:174-203",
            "fr": "core/src/common/mont/tests/main.cu:238-252,369-383,527-532",
        },
        "curve": {k: hexlimbs(curve[k]) for k in
                  ("p1_x", "p1_y", "p2_x", "p2_y", "pr_x", "pr_y", "pr100_x", "pr100_y",
                   "p1r128_x", "p1r128_y")},
        "fr": {ns: {k: hexlimbs(v) for k, v in d.items()} for ns, d in parse_namespaces(mont_src).items()},
    }
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1, sort_keys=True)

    # ---- MSM golden cases, outputs from the reference's own arithmetic.
    cases = []
    r_minus_1 = O.int_to_limbs(O.to_mont(O.R_MOD - 1, O.R_MOD))
    one_m = O.int_to_limbs(O.to_mont(1, O.R_MOD))

    def add_case(name, pts, sc):
        pts = np.ascontiguousarray(pts, dtype=np.uint32).reshape(-1, 16)
        sc = np.ascontiguousarray(sc, dtype=np.uint32).reshape(-1, 8)
        out = O.ref_msm_naive(pts, sc)
        cases.append({"name": name, "n": int(pts.shape[0]), "points": rows_hex(pts),
                      "scalars": rows_hex(sc), "result": "".join(hexlimbs(out))})

    pts = O.gen_points(256, seed=0)
    add_case("uniform_n1", pts[:1], O.gen_scalars(1, seed=0, stream=1))
    add_case("uniform_n7", pts[:7], O.gen_scalars(7, seed=0, stream=1))
    add_case("uniform_n64", pts[:64], O.gen_scalars(64, seed=0, stream=1))
    add_case("uniform_n256", pts, O.gen_scalars(256, seed=0, stream=1))
    add_case("skewed_n256", pts, O.gen_scalars(256, seed=0, stream=3, dist=O.DIST_SKEWED))
    add_case("zero_scalars_n16", pts[:16], np.zeros((16, 8), np.uint32))
    add_case("scalar_one_n1", pts[:1], one_m[None, :])
    neg = O.point_op(O.PT_NEG, pts[:1])
    add_case("p_and_minus_p", np.concatenate([pts[:1], neg]), np.stack([one_m, one_m]))
    rep = np.repeat(pts[:1], 33, axis=0)
    add_case("repeated_point_n33", rep, O.gen_scalars(33, seed=0, stream=4))
    add_case("scalar_r_minus_1_n8", pts[:8], np.repeat(r_minus_1[None, :], 8, axis=0))
    ident = pts[:32].copy()
    ident[::5] = 0
    add_case("identity_points_n32", ident, O.gen_scalars(32, seed=0, stream=5))
    mixed = O.gen_scalars(64, seed=0, stream=6)
    mixed[::3] = 0
    mixed[1::7] = one_m
    mixed[2::11] = r_minus_1
    add_case("mixed_edges_n64", pts[:64], mixed)
    with open(os.path.join(HERE, "msm_golden.json"), "w") as f:
        json.dump({"source": "outputs computed with oracle/_ref/libref_bn254.so (reference host arithmetic)",
                   "cases": cases}, f, indent=0)
    bls_cases()

    gen = {
        "srs_points_seed0_first4": rows_hex(O.gen_points(4, seed=0)),
        "srs_r_seed0_first4": rows_hex(O.gen_scalars(4, seed=0, stream=0, mont=False)),
        "uniform_seed0_stream1_first4_mont": rows_hex(O.gen_scalars(4, seed=0, stream=1)),
        "skewed_seed0_stream2_first32_canonical": rows_hex(
            O.gen_scalars(32, seed=0, stream=2, dist=O.DIST_SKEWED, mont=False)),
    }
    with open(os.path.join(HERE, "generators.json"), "w") as f:
        json.dump(gen, f, indent=1)
    print("wrote kat.json, msm_golden.json, generators.json")


def bls_cases() -> None:
    C = O.BLS12381
    cases = []
    r_minus_1 = O.int_to_limbs(O.to_mont(O.R_BLS - 1, O.R_BLS))
    one_m = O.int_to_limbs(O.to_mont(1, O.R_BLS))

    def add_case(name, pts, sc):
        pts = np.ascontiguousarray(pts, dtype=np.uint32).reshape(-1, 24)
        sc = np.ascontiguousarray(sc, dtype=np.uint32).reshape(-1, 8)
        out = O.ref_msm_naive(pts, sc, curve=C)
        cases.append({"name": name, "n": int(pts.shape[0]), "points": rows_hex(pts),
                      "scalars": rows_hex(sc), "result": "".join(hexlimbs(out))})

    pts = O.gen_points(128, seed=0, curve=C)
    add_case("uniform_n1", pts[:1], O.gen_scalars(1, seed=0, stream=1, curve=C))
    add_case("uniform_n9", pts[:9], O.gen_scalars(9, seed=0, stream=1, curve=C))
    add_case("uniform_n128", pts, O.gen_scalars(128, seed=0, stream=1, curve=C))
    add_case("skewed_n128", pts, O.gen_scalars(128, seed=0, stream=3, dist=O.DIST_SKEWED, curve=C))
    add_case("zero_scalars_n8", pts[:8], np.zeros((8, 8), np.uint32))
    neg = O.point_op(O.PT_NEG, pts[:1], curve=C)
    add_case("p_and_minus_p", np.concatenate([pts[:1], neg]), np.stack([one_m, one_m]))
    add_case("repeated_point_n17", np.repeat(pts[:1], 17, axis=0), O.gen_scalars(17, seed=0, stream=4, curve=C))
    add_case("scalar_r_minus_1_n4", pts[:4], np.repeat(r_minus_1[None, :], 4, axis=0))
    ident = pts[:24].copy()
    ident[::5] = 0
    add_case("identity_points_n24", ident, O.gen_scalars(24, seed=0, stream=5, curve=C))
    mixed = O.gen_scalars(48, seed=0, stream=6, curve=C)
    mixed[::3] = 0
    mixed[1::7] = one_m
    mixed[2::11] = r_minus_1
    add_case("mixed_edges_n48", pts[:48], mixed)
    with open(os.path.join(HERE, "msm_golden_bls12381.json"), "w") as f:
        json.dump({"source": "outputs computed with oracle/_ref/libref_bn254.so ref_bls_msm_naive "
                             "(reference host arithmetic, BLS12-381 G1)", "cases": cases}, f, indent=0)
    gen = {
        "srs_points_seed0_first4": rows_hex(O.gen_points(4, seed=0, curve=C)),
        "srs_r_seed0_first4": rows_hex(O.gen_scalars(4, seed=0, stream=0, mont=False, curve=C)),
        "uniform_seed0_stream1_first4_mont": rows_hex(O.gen_scalars(4, seed=0, stream=1, curve=C)),
        "skewed_seed0_stream2_first32_canonical": rows_hex(
            O.gen_scalars(32, seed=0, stream=2, dist=O.DIST_SKEWED, mont=False, curve=C)),
    }
    with open(os.path.join(HERE, "generators_bls12381.json"), "w") as f:
        json.dump(gen, f, indent=1)


if __name__ == "__main__":
    default_root = os.environ.get("REF_ROOT") or os.path.abspath(os.path.join(HERE, "..", "..", "..", "reference"))
    main(sys.argv[1] if len(sys.argv) > 1 else default_root)
