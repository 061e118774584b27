"""Builds lib/libcuwaves.so from csrc/ with nvcc for sm_100a."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = ["capi.cu", "fft.cu", "gemm.cu", "ortho.cu", "tc.cu", "serve.cu", "tune.cu", "restart.cu"]
OUT = os.path.join(HERE, "lib", "libcuwaves.so")


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(verbose: bool = False, force: bool = False) -> str:
    srcs = [os.path.join(HERE, "csrc", s) for s in SRC]
    deps = srcs + [os.path.join(HERE, "csrc", "cuwaves_internal.cuh"), os.path.join(HERE, "csrc", "tc_sm100.cuh"),
                   os.path.join(HERE, "csrc", "tc_pipe.cuh"),
                   os.path.join(os.path.dirname(HERE), "include", "cuwaves.h")]
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(d) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [nvcc(), "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
           "-Xcompiler", "-fPIC", "-shared", "-o", OUT] + srcs
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose:
        sys.stderr.write(r.stderr)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force=True)
    print(OUT)
