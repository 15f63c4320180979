"""Builds the in-tree CUDA library ``rtrace_b200/_lib/librtrace_b200.so``.

The device code is compiled for sm_100a only, with IEEE double arithmetic
in source order (``-fmad=false`` on the device, ``-ffp-contract=off`` on the
host): the renderer's results must match the reference's double-precision
CPU arithmetic bit for bit.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "librtrace_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "-Xptxas", "-v",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build rtrace_b200")


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cpp", ".cuh", ".hpp"))] + [
        os.path.join(HERE, "..", "include", "rtrace_gpu.h")]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force=False, verbose=False):
    """Compile the library if any source is newer than it; returns its path."""
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    cmds, objs = [], []
    for src in sorted(os.listdir(CSRC)):
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src + ".o")
        if src.endswith(".cu"):
            cmds.append([nvcc, *NVCC_FLAGS, "-c", path, "-o", obj])
        elif src.endswith(".cpp"):
            cmds.append(["g++", *CXX_FLAGS, "-c", path, "-o", obj])
        else:
            continue
        objs.append(obj)
    # translation units compile independently: one process each, in parallel
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        results = list(pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    log = []
    for cmd, r in zip(cmds, results):
        log.append(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("compile failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp, *objs,
           "-Xcompiler", "-fPIC", "-lz"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    os.replace(tmp, LIB)
    if verbose:
        sys.stdout.write("".join(log))
    with open(os.path.join(BUILD_DIR, "ptxas.log"), "w") as f:
        f.write("".join(log))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
