"""The no-allocation projections entry point (cuwaves_projections_noalloc).

It serves callers that cannot allocate device memory themselves, e.g. a host
code that owns a fixed device pool or a plug-in inside another program's
stream capture.  The test drives it through the C ABI with buffers it owns,
twice in a row (the static scratch keeps the previous call's contents), and
compares each result with the regular entry point cuwaves_projections at the
projection tolerance of the parity tests (1e-10 relative).  This file is
collected last so that a failure here stops a run only after all other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import cuwaves  # noqa: E402
from cuwaves import systems  # noqa: E402


def _device_inputs(inp, w):
    import torch

    dev = torch.device("cuda")
    psi = torch.from_numpy(w.download_psi(cuwaves.CUW_PSI0)).to(dev).contiguous()  # (nbh, ngl): ldg = ngl
    ylm = torch.from_numpy(np.ascontiguousarray(inp["ylm"])).to(dev)
    pro = torch.from_numpy(np.ascontiguousarray(inp["pro"])).to(dev)
    ph = inp["gvec"] @ inp["r0"].T  # (ngl, nat)
    eigr = torch.from_numpy(np.ascontiguousarray(np.exp(-1j * ph).T)).to(dev)  # (nat, ngl) == EIGR(ngl,nat)
    desc, ibare0 = [], np.cumsum([0] + list(inp["lnx"]))
    for a, s in enumerate(inp["isp"].tolist()):
        for ln, l in enumerate(inp["lox"][s - 1]):
            for m in range(2 * l + 1):
                desc.append((a, int(ibare0[s - 1]) + ln, l * l + m, l))
    pdesc = torch.tensor(np.array(desc, dtype=np.int32).ravel(), device=dev)
    return psi, pdesc, ylm, pro, eigr, len(desc)


def test_projections_noalloc_matches_regular_entry_point():
    import torch

    inp = systems.build_inputs(systems.named_system("Si8"))
    w = cuwaves.open_waves(inp).setup().initialize()
    want = w.get_proj()  # cuwaves_projections of PSI0 at R(0)
    psi, pdesc, ylm, pro, eigr, npro = _device_inputs(inp, w)
    lib = cuwaves.load_library()
    f = lib.cuwaves_projections_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    stream = torch.cuda.current_stream()
    for call in range(2):
        out = torch.full((npro, inp["nbh"]), float("nan"), dtype=torch.complex128, device="cuda")
        rc = f(inp["ngl"], inp["ngl"], inp["nbh"], inp["nat"], npro, psi.data_ptr(), pdesc.data_ptr(),
               ylm.data_ptr(), pro.data_ptr(), eigr.data_ptr(), float(inp["omega"]), out.data_ptr(),
               stream.cuda_stream)
        assert rc == 0, f"call {call}: status {rc}"
        stream.synchronize()
        got = out.cpu().numpy()
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err < 1e-10, f"call {call}: relative error {err:.3e}"
    # sizes beyond the static scratch are refused before any launch
    rc = f(inp["ngl"], inp["ngl"], 1 << 12, inp["nat"], 1 << 12, psi.data_ptr(), pdesc.data_ptr(),
           ylm.data_ptr(), pro.data_ptr(), eigr.data_ptr(), 1.0, out.data_ptr(), stream.cuda_stream)
    assert rc == 1
    w.close()
