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


def _entry():
    lib = cuwaves.load_library()
    f = lib.cuwaves_projections_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    return f


def test_projections_noalloc_matches_regular_entry_point():
    import torch

    inp = systems.build_inputs(systems.named_system("Si8"))
    w = cuwaves.open_waves(inp).setup().initialize()
    want = w.get_proj()  # cuwaves_projections of PSI0 at R(0)
    psi, pdesc, ylm, pro, eigr, npro = _device_inputs(inp, w)
    f = _entry()
    stream = torch.cuda.current_stream()
    # the same bands at a padded leading dimension (ldg = ngl + 7); the padding
    # holds values that would spoil every sum if the kernel read them
    ngl, nbh, ldg = inp["ngl"], inp["nbh"], inp["ngl"] + 7
    psi_pad = torch.full((nbh, ldg), 1e30 + 1e30j, dtype=torch.complex128, device="cuda")
    psi_pad[:, :ngl] = psi
    outs = [torch.full((npro, nbh), float("nan"), dtype=torch.complex128, device="cuda") for _ in range(4)]
    torch.cuda.synchronize()
    free = []
    for call, (x, ld) in enumerate([(psi, ngl), (psi, ngl), (psi_pad, ldg), (psi_pad, ldg)]):
        out = outs[call]
        rc = f(ngl, ld, nbh, inp["nat"], npro, x.data_ptr(), pdesc.data_ptr(), ylm.data_ptr(), pro.data_ptr(),
               eigr.data_ptr(), float(inp["omega"]), out.data_ptr(), stream.cuda_stream)
        assert rc == 0, f"call {call}: status {rc}"
        stream.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        got = out.cpu().numpy()
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err < 1e-10, f"call {call} (ldg {ld}): relative error {err:.3e}"
    # after the first call (which commits the static array) no call changes the
    # device memory in use
    assert free[1:] == free[:1] * 3, free
    # sizes beyond the static scratch are refused before any launch
    rc = f(ngl, ngl, 1 << 12, inp["nat"], 1 << 12, psi.data_ptr(), pdesc.data_ptr(),
           ylm.data_ptr(), pro.data_ptr(), eigr.data_ptr(), 1.0, outs[0].data_ptr(), stream.cuda_stream)
    assert rc == 1
    w.close()


def test_projections_noalloc_single_split():
    """nbh*npro above half the static array leaves room for one split only: the
    whole G sum then runs in one K range.  Checked against the contraction
    PROJ(b,p) = gweight sum_G conj(PRO(G,p)) psi(G,b) with
    PRO(G,p) = Y_lm(G) P(G) (-i)^l exp(-iG.R_a), formed in numpy in FP64."""
    import torch

    rng = np.random.default_rng(11)
    ngl, ldg, nbh, nat = 2000, 2016, 264, 64
    lox = [0, 0, 1, 1]  # two s and two p projectors per atom: 8 per atom
    desc = []
    for a in range(nat):
        for ln, l in enumerate(lox):
            for m in range(2 * l + 1):
                desc.append((a, ln, l * l + m, l))
    npro = len(desc)
    assert nbh * npro > (1 << 17) and nbh * npro <= (1 << 18)
    psi = (rng.standard_normal((nbh, ldg)) + 1j * rng.standard_normal((nbh, ldg))) * 0.1
    ylm = rng.standard_normal((4, ngl))  # YLM(ngl, 4) column-major
    pro = rng.standard_normal((4, ngl))
    eigr = np.exp(-1j * rng.uniform(0, 2 * np.pi, (nat, ngl)))
    gweight = 1.7
    want = np.empty((npro, nbh), dtype=np.complex128)
    for p, (a, col, lm, l) in enumerate(desc):
        prog = ylm[lm] * pro[col] * (-1j) ** l * eigr[a]
        want[p] = gweight * (np.conj(prog)[None, :] * psi[:, :ngl]).sum(axis=1)
    dev = torch.device("cuda")
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         dict(psi=psi, ylm=ylm, pro=pro, eigr=eigr).items()}
    pdesc = torch.tensor(np.array(desc, dtype=np.int32).ravel(), device=dev)
    f = _entry()
    stream = torch.cuda.current_stream()
    for call in range(2):
        out = torch.full((npro, nbh), float("nan"), dtype=torch.complex128, device=dev)
        rc = f(ngl, ldg, nbh, nat, npro, t["psi"].data_ptr(), pdesc.data_ptr(), t["ylm"].data_ptr(),
               t["pro"].data_ptr(), t["eigr"].data_ptr(), gweight, out.data_ptr(), stream.cuda_stream)
        assert rc == 0, f"call {call}: status {rc}"
        stream.synchronize()
        err = np.abs(out.cpu().numpy() - want).max() / np.abs(want).max()
        assert err < 1e-10, f"call {call}: relative error {err:.3e}"
