"""The autotuner (cuwaves_autotune): FFT band batch and split-K factors timed
on the handle's own data.  No reference counterpart (FFTW's planner picks the
reference's FFT plans)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import cuwaves  # noqa: E402
from cuwaves import CUW_PREC_FP64, CUW_PREC_MIXED, systems  # noqa: E402


@pytest.fixture(scope="module")
def inputs():
    return {"H2O2": systems.build_inputs(systems.water_box(2, box=10.0, lattice=(2, 1, 1), epw_psi_ry=25.0,
                                                            grid=(32, 32, 32)))}


@pytest.mark.parametrize("prec", [CUW_PREC_FP64, CUW_PREC_MIXED])
def test_autotune_keeps_results_and_caches_by_shape(inputs, prec):
    """The tuned launch shapes change summation orders only: energies and
    forces stay within rounding-level distance of the untuned run; a second
    handle of the same shape takes the choice from the table."""
    inp = inputs["H2O2"]
    ws = [cuwaves.open_waves(inp, precision=prec).setup().initialize() for _ in range(3)]
    t1 = ws[1].autotune()
    t2 = ws[2].autotune()
    assert t1["fft_batch"] >= 1 and t1["split_proj"] > 0 and t1["split_gram"] > 0
    assert t2["cached"] == 1.0 and t2["fft_batch"] == t1["fft_batch"]
    tol_e, tol_f = (1e-9, 1e-8) if prec == CUW_PREC_FP64 else (1e-5, 1e-5)
    for _ in range(4):
        (o0, f0), (o1, f1) = ws[0].cp_step(move_atoms=True), ws[1].cp_step(move_atoms=True)
        assert abs(o0[0] - o1[0]) < tol_e and np.abs(f0 - f1).max() < tol_f
    for w in ws:
        w.close()
