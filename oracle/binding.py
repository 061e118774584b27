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


def blas_path():
    """The OpenBLAS bundled with scipy (its CBLAS ZGEMM), or None.  The
    reference's fast build links a BLAS for the ZGEMMs of LIB$SCALARPRODUCTC8
    and LIB$ADDPRODUCTC8; the oracle uses this one when it is there
    (CPWAVES_ORACLE_BLAS=0 keeps the plain loops)."""
    if os.environ.get("CPWAVES_ORACLE_BLAS", "1") == "0":
        return None
    import glob
    import importlib.util

    spec = importlib.util.find_spec("scipy")
    if spec is None or not spec.submodule_search_locations:
        return None
    libs = os.path.join(os.path.dirname(list(spec.submodule_search_locations)[0]), "scipy.libs")
    found = sorted(glob.glob(os.path.join(libs, "libscipy_openblas-*.so")))
    return found[0] if found else None


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
        _lib.orc_use_blas.argtypes = [C.c_char_p]
        _lib.orc_use_blas.restype = C.c_int
        _lib.orc_blas_in_use.restype = C.c_int
        path = blas_path()
        if path:
            _lib.orc_use_blas(path.encode())
    return _lib


def blas_in_use() -> bool:
    return bool(library().orc_blas_in_use())


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
