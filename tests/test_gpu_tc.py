"""Split-precision tensor-core product (tcgen05, kind::tf32, three terms).

cuwaves_tc_gemm_check computes C = A B^T from FP64 operands split into tf32
pairs, accumulated in fp32 in tensor memory and drained after every K = 8
step.  The result is compared with the FP64 product; three-term tf32 products
carry about 21 significant bits, so the error bound is stated relative to the
largest |C| (2e-6), ragged sizes included.  The signed mean error (the bias of
the tensor core's truncating accumulation) must stay below 1e-7 of mean |C|.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import cuwaves  # noqa: E402


@pytest.mark.parametrize("m,n,k", [(128, 128, 32), (300, 200, 1000), (77, 19, 4099), (512, 128, 8000)])
def test_tf32x3_gemm_matches_fp64(m, n, k):
    import torch

    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a = rng.normal(size=(m, k))
    b = rng.normal(size=(n, k))
    want = a @ b.T
    lib = cuwaves.load_library()
    f = lib.cuwaves_tc_gemm_check
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b).cuda()
    dc = torch.full((m, n), float("nan"), dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    rc = f(m, n, k, da.data_ptr(), db.data_ptr(), dc.data_ptr(), err.data_ptr(), s.cuda_stream)
    assert rc == 0
    s.synchronize()
    assert int(err.item()) == 0, "a bounded wait in the kernel ran out"
    got = dc.cpu().numpy()
    rel = np.abs(got - want).max() / np.abs(want).max()
    bias = float(np.sum((got - want) * np.sign(want)) / np.sum(np.abs(want)))
    print(f"tf32x3 {m}x{n}x{k}: max error / max |C| = {rel:.3e}, bias {bias:+.2e}")
    # one-term tf32 would give ~1e-3; three terms must reach fp32 level
    assert rel < 2e-6, rel
    assert abs(bias) < 1e-7, bias
