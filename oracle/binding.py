"""ctypes binding of the CPU oracle (test infrastructure only).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU legs to check or
time the CUDA engine; the product never imports it.  The oracle exports the
C ABI of include/cuwaves.h under the prefix orc_.
"""
import ctypes as C
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "cp-paw_b200"))

from cuwaves.capi import Waves, bind  # noqa: E402

LIB = os.path.join(HERE, "liboracle_cpwaves.so")
_fns = None
_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "cpwaves_oracle.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "liboracle_cpwaves.so"])
    return LIB


def library() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB)
        _lib.orc_mslng.argtypes = [C.POINTER(C.c_int)]
        _lib.orc_mslng.restype = C.c_double
        for name in ("orc_getig",):
            getattr(_lib, name).restype = C.c_int
        _lib.orc_max_threads.restype = C.c_int
    return _lib


def fns() -> dict:
    global _fns
    if _fns is None:
        _fns = bind(library(), "orc_")
    return _fns


def open_oracle(inputs: dict, threads: int = 0) -> Waves:
    w = Waves(fns(), inputs)
    if threads and "set_threads" in w._f:
        w._f["set_threads"](w.h, threads)
    return w
