"""Builds lib/libcuwaves.so from csrc/ with nvcc for sm_100a.

Each source compiles to its own object (in parallel, under lib/obj/), and the
objects link into one shared library; an object is rebuilt when its source or
any shared header is newer.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = ["capi.cu", "fft.cu", "gemm.cu", "ortho.cu", "tc.cu", "serve.cu", "tune.cu", "restart.cu", "vofrho.cu"]
HDR = ["cuwaves_internal.cuh", "tc_sm100.cuh", "tc_pipe.cuh"]
OUT = os.path.join(HERE, "lib", "libcuwaves.so")
OBJ = os.path.join(HERE, "lib", "obj")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _sources():
    return [s for s in SRC if os.path.exists(os.path.join(HERE, "csrc", s))]


def build(verbose: bool = False, force: bool = False) -> str:
    srcs = _sources()
    hdrs = [os.path.join(HERE, "csrc", h) for h in HDR] + [
        os.path.join(os.path.dirname(HERE), "include", "cuwaves.h")]
    hdr_time = max(os.path.getmtime(h) for h in hdrs)
    os.makedirs(OBJ, exist_ok=True)

    def obj_of(s):
        return os.path.join(OBJ, s[:-3] + ".o")

    def stale(s):
        o = obj_of(s)
        return force or not os.path.exists(o) or os.path.getmtime(o) < max(
            hdr_time, os.path.getmtime(os.path.join(HERE, "csrc", s)))

    todo = [s for s in srcs if stale(s)]
    if not todo and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(obj_of(s)) for s in srcs):
        return OUT

    def compile_one(s):
        cmd = [nvcc()] + FLAGS + (["-Xptxas=-v"] if verbose else []) + [
            "-c", os.path.join(HERE, "csrc", s), "-o", obj_of(s)]
        return s, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
        results = list(ex.map(compile_one, todo))
    failed = False
    for s, r in results:
        if r.returncode != 0:
            sys.stderr.write(f"== {s}\n" + r.stdout + r.stderr)
            failed = True
        elif verbose:
            sys.stderr.write(f"== {s}\n" + r.stderr)
    if failed:
        raise RuntimeError("nvcc failed")
    cmd = [nvcc()] + FLAGS + ["-shared", "-o", OUT] + [obj_of(s) for s in srcs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv or "-v" in sys.argv)
    print(OUT)
