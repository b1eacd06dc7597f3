"""Build libimpeller_msm.so (sm_100a only) in-tree.

  python -m impeller_b200.build [--verbose] [--ptxas-v]

Every .cu under csrc/ is compiled with
  nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo
and linked into impeller_b200/libimpeller_msm.so with the CUDA runtime linked
statically, so the library loads on any box with the same driver.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libimpeller_msm.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-I" + os.path.join(ROOT, "include"),
           "-Wno-deprecated-gpu-targets"]

SOURCES = ["engine.cu", "abi.cu", "aux_kernels.cu", "noalloc.cu", "serve.cu", "ntt.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps() -> list[str]:
    files = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h", ".cpp", ".inc")):
                files.append(os.path.join(d, f))
    return files


def write_default_table() -> None:
    """csrc/autotune_default.inc from autotune_table.json (rewritten only when it changes)."""
    sys.path.insert(0, ROOT)
    from impeller_b200 import autotune
    text = autotune.c_include()
    path = os.path.join(CSRC, "autotune_default.inc")
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as f:
            f.write(text)


def build(verbose: bool = False, ptxas_v: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    write_default_table()
    deps = _deps()
    if not force and not _stale(LIB, deps + [os.path.abspath(__file__)]):
        return LIB
    cc = nvcc()
    extra = ["-Xptxas", "-v"] if ptxas_v else []

    def compile_one(src: str) -> tuple[str, str]:
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        cmd = [cc, *ARCH, *NVFLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return obj, r.stdout + r.stderr

    # an object is rebuilt when its source, a header or this script is newer
    headers = [d for d in deps if not d.endswith(".cu")] + [os.path.abspath(__file__)]
    todo = [src for src in SOURCES
            if force or _stale(os.path.join(OBJ, src.replace(".cu", ".o")), [os.path.join(CSRC, src)] + headers)]
    with cf.ThreadPoolExecutor(max_workers=max(1, len(todo))) as ex:
        results = list(ex.map(compile_one, todo))
    if verbose or ptxas_v:
        for _, log in results:
            if log.strip():
                print(log)
    objs = [os.path.join(OBJ, src.replace(".cu", ".o")) for src in SOURCES]
    tmp = LIB + ".tmp"
    cmd = [cc, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs, "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


SHIM_DIR = os.path.join(HERE, "lib")


CURVE_NAMES = ("bn254", "bls12381")


def build_shim(window_size: int, target_window: int, debug: bool = False, curve: int = 0) -> str:
    """lib/libmsm_{curve}_{c}_{alpha}_{debug}.so forwarding to libimpeller_msm.so
    (rpath $ORIGIN/..), the reference's per-configuration library name."""
    core = build()
    os.makedirs(SHIM_DIR, exist_ok=True)
    name = f"libmsm_{CURVE_NAMES[curve]}_{window_size}_{target_window}_{'true' if debug else 'false'}.so"
    out = os.path.join(SHIM_DIR, name)
    src = os.path.join(CSRC, "shim", "msm_shim.c")
    if not _stale(out, [src, core, os.path.join(ROOT, "include", "impeller_msm.h")]):
        return out
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc())), "include")
    cmd = ["gcc", "-O2", "-shared", "-fPIC", f"-DMSM_WINDOW_SIZE={int(window_size)}",
           f"-DMSM_TARGET_WINDOWS={int(target_window)}", f"-DMSM_DEBUG={1 if debug else 0}",
           f"-DMSM_CURVE_ID={int(curve)}",
           "-I" + os.path.join(ROOT, "include"), "-I" + cuda_inc, src, "-o", out + ".tmp",
           "-L" + HERE, "-limpeller_msm", "-Wl,-rpath,$ORIGIN/.."]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"shim build failed:\n{r.stdout}\n{r.stderr}")
    os.replace(out + ".tmp", out)
    return out


def ntt_library() -> str:
    """lib/libntt.so, the name the reference's NTT operator loads
    (core/src/ntt.rs:23, 98-106): a link to libimpeller_msm.so, which exports
    ssip_ntt, ssip_precompute, recompute_ntt, gen_pq_omegas and
    distribute_powers for BN254 Fr (the reference's default NTT_FIELD)."""
    build()
    os.makedirs(SHIM_DIR, exist_ok=True)
    out = os.path.join(SHIM_DIR, "libntt.so")
    if not os.path.islink(out):
        if os.path.exists(out):
            os.remove(out)
        os.symlink(os.path.join("..", os.path.basename(LIB)), out)
    return out


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_v="--ptxas-v" in sys.argv, force="--force" in sys.argv)
    print(LIB)
