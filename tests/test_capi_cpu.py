"""The C ABI library loads here (no GPU) and exports every entry point that
include/cuwaves.h declares; argument validation happens before any device call."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            with open(os.path.join(ROOT, "include", fn)) as f:
                names |= set(re.findall(r"^\s*int\s+(cuwaves_\w+)\s*\(", f.read(), flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol(engine_lib):
    lib = engine_lib.load_library()
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_abi(engine_lib):
    from cuwaves.capi import OPTIONAL, SIGNATURES
    from cuwaves.serve import _bind

    bound = {"cuwaves_" + n for n in list(SIGNATURES) + list(OPTIONAL)}
    bound |= {"cuwaves_server_" + n for n in _bind()}
    assert set(declared_symbols()) <= bound


def test_oracle_exports_the_same_abi(oracle):
    lib = oracle.library()
    for n in declared_symbols():
        if n.startswith("cuwaves_server_") or n.startswith("cuwaves_batch_"):  # runtime over the ABI
            continue
        if n in ("cuwaves_set_async", "cuwaves_synchronize", "cuwaves_set_timing", "cuwaves_get_timing",
                 "cuwaves_get_stream", "cuwaves_get_ortho_stats", "cuwaves_projections_noalloc",
                 "cuwaves_tc_gemm_check", "cuwaves_set_option", "cuwaves_get_graph_stats",
                 "cuwaves_autotune"):  # device-only entry points
            continue
        assert hasattr(lib, n.replace("cuwaves_", "orc_")), n


def test_invalid_dims_rejected_without_device(engine_lib):
    from cuwaves.capi import Dims

    lib = engine_lib.load_library()
    f = lib.cuwaves_create
    f.argtypes = [C.POINTER(Dims), C.POINTER(C.c_void_p)]
    h = C.c_void_p()
    lib.cuwaves_last_error.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
    buf = C.create_string_buffer(256)

    def why():
        lib.cuwaves_last_error(None, buf, 256)  # the thread's last failed create
        return buf.value.decode()

    d = Dims()  # all zero: invalid
    assert f(C.byref(d), C.byref(h)) == 1  # CUW_ERR_ARG
    assert why() == "invalid dimensions"
    d.ngl, d.ndim, d.nb, d.nbh, d.tinv = 100, 1, 3, 2, 1  # odd NB with super wave functions
    d.nr1 = d.nr2 = d.nr3 = 8
    d.nsp, d.lmx = 1, 1
    d.lnx[0] = 1
    isp = (C.c_int * 1)(1)
    d.nat = 1
    d.isp = C.cast(isp, C.POINTER(C.c_int))
    assert f(C.byref(d), C.byref(h)) == 6  # CUW_ERR_UNSUPPORTED
    assert "even band count" in why()
    d.nb, d.nbh = 4, 2
    rc = f(C.byref(d), C.byref(h))
    # valid dims: without a CUDA device the engine refuses (no host fallback)
    import torch

    if not torch.cuda.is_available():
        assert rc == 2  # CUW_ERR_CUDA
        assert why() == "no CUDA device"
    else:
        assert rc == 0
        lib.cuwaves_destroy.argtypes = [C.c_void_p]
        lib.cuwaves_destroy(h)


def test_server_admission_rules_without_device(engine_lib):
    """Submission validates and copies on the host; a request whose estimated
    device memory exceeds the whole budget is refused (CUW_ERR_NOMEM), and an
    idle server shuts down cleanly."""
    from cuwaves import systems
    from cuwaves.capi import WavesError
    from cuwaves.serve import Server

    inp = systems.build_inputs(systems.molecule_box("Si2", box=12.0))
    srv = Server(hbm_budget=1 << 20, workers=2)  # 1 MiB: nothing fits
    with pytest.raises(WavesError) as e:
        srv.submit(inp, nsteps=0)
    assert e.value.code == 8
    bad = dict(inp)
    bad["isp"] = np.full_like(np.asarray(inp["isp"]), 7)  # species index out of range
    with pytest.raises(WavesError) as e:
        srv.submit(bad, nsteps=0)
    assert e.value.code == 1
    st = srv.stats()
    assert st["completed"] == 0 and st["in_system"] == 0 and st["peak_bytes"] == 0
    srv.close()
    with pytest.raises(WavesError):
        Server(hbm_budget=0)
