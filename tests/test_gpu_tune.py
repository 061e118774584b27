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


@pytest.mark.parametrize("prec", [CUW_PREC_FP64, CUW_PREC_MIXED])
def test_fft_plan_variants_agree(inputs, prec, oracle):
    """Every FFT plan variant the autotuner can pick gives H|psi> of the
    oracle (FP64: 1e-10 relative; FP32 transforms: 1e-5), on a grid with
    compiled kernels; the tuner reports the variant it kept; a grid without
    compiled kernels refuses variants other than 0."""
    inp = inputs["H2O2"]
    w = cuwaves.open_waves(inp, precision=prec).setup().initialize()
    cpu = oracle.open_oracle(inp).setup()
    for which in (cuwaves.CUW_PSI0, cuwaves.CUW_PSIM):
        cpu.upload_psi(which, w.download_psi(which))
    cpu.set_proj(w.get_proj())
    cpu.hpsi()
    ref = cpu.download_psi(cuwaves.CUW_HPSI)
    tol = 1e-10 if prec == CUW_PREC_FP64 else 1e-5
    for v in range(3):
        w.set_option(cuwaves.CUW_OPT_FFT_VARIANT, v)
        w.hpsi()
        got = w.download_psi(cuwaves.CUW_HPSI)
        err = float(np.abs(got - ref).max() / np.abs(ref).max())
        assert err < tol, f"variant {v}: {err:.2e}"
    t = w.autotune()
    assert t["fft_variant"] in (0.0, 1.0, 2.0)
    w.close()
    cpu.close()
    odd = systems.build_inputs(systems.water_box(2, box=10.0, lattice=(2, 1, 1), epw_psi_ry=25.0,
                                                 grid=(30, 30, 30)))
    w2 = cuwaves.open_waves(odd, precision=prec).setup()
    w2.set_option(cuwaves.CUW_OPT_FFT_VARIANT, 0)
    with pytest.raises(cuwaves.WavesError) as e:
        w2.set_option(cuwaves.CUW_OPT_FFT_VARIANT, 1)
    assert e.value.code == 6
    w2.close()


def test_contraction_tile_families(inputs):
    """The two tile families of the mixed path's contractions: split-tf32
    tcgen05 tiles (128 x 128 x 8) and FP64 DMMA tiles (64 x 64 x 4).  A CP step
    on either agrees with the FP64 handle within the mixed path's tolerance,
    the DMMA tiles (FP64 products, FP32 transforms) closer than that; FP64
    handles refuse the tcgen05 family; the autotuner times both and keeps the
    faster."""
    inp = inputs["H2O2"]
    ref = cuwaves.open_waves(inp, precision=CUW_PREC_FP64).setup().initialize()
    with pytest.raises(cuwaves.WavesError):
        ref.set_option(cuwaves.CUW_OPT_CONTRACTION_TILES, 0)
    ref.set_option(cuwaves.CUW_OPT_CONTRACTION_TILES, 1)
    state = (ref.download_psi(cuwaves.CUW_PSI0), ref.download_psi(cuwaves.CUW_PSIM), ref.get_proj())
    o_ref, f_ref = ref.cp_step(move_atoms=True)
    errs = {}
    for fam in (0, 1):
        w = cuwaves.open_waves(inp, precision=CUW_PREC_MIXED).setup()
        w.upload_psi(cuwaves.CUW_PSI0, state[0])
        w.upload_psi(cuwaves.CUW_PSIM, state[1])
        w.set_proj(state[2])
        w.set_option(cuwaves.CUW_OPT_CONTRACTION_TILES, fam)
        o, f = w.cp_step(move_atoms=True)
        errs[fam] = (abs(o[0] - o_ref[0]) / inp["nat"], float(np.abs(f - f_ref).max()))
        w.close()
    for fam, (de, df) in errs.items():
        assert de < 1e-6 and df < 1e-4, (fam, de, df)
    w = cuwaves.open_waves(inp, precision=CUW_PREC_MIXED).setup().initialize()
    t = w.autotune()
    assert t["dmma_tiles"] in (0.0, 1.0) and t["tc_tiles_ms"] > 0 and t["dmma_tiles_ms"] > 0
    assert t["dmma_tiles"] == float(t["dmma_tiles_ms"] < t["tc_tiles_ms"])
    w.close()
    ref.close()


@pytest.mark.parametrize("prec", [CUW_PREC_FP64, CUW_PREC_MIXED])
def test_fft_shuffle_variant(prec, oracle):
    """Plan variant 3 (64^3 grids): the 8 x 8 exchange of the 64-point z
    transforms by warp shuffles among a column's lanes instead of shared
    memory gives H|psi> of the oracle (FP64: 1e-10 relative; FP32 transforms:
    1e-5), the same as variant 0 to rounding; a grid of another size refuses
    it."""
    inp = systems.build_inputs(systems.si_cell(1, grid=(64, 64, 64), epw_psi_ry=30.0, name="Si8-64"))
    w = cuwaves.open_waves(inp, precision=prec).setup().initialize()
    cpu = oracle.open_oracle(inp).setup()
    for which in (cuwaves.CUW_PSI0, cuwaves.CUW_PSIM):
        cpu.upload_psi(which, w.download_psi(which))
    cpu.set_proj(w.get_proj())
    cpu.hpsi()
    ref = cpu.download_psi(cuwaves.CUW_HPSI)
    tol = 1e-10 if prec == CUW_PREC_FP64 else 1e-5
    got = {}
    for v in (0, 3):
        w.set_option(cuwaves.CUW_OPT_FFT_VARIANT, v)
        w.hpsi()
        got[v] = w.download_psi(cuwaves.CUW_HPSI)
        err = float(np.abs(got[v] - ref).max() / np.abs(ref).max())
        assert err < tol, f"variant {v}: {err:.2e}"
    assert float(np.abs(got[3] - got[0]).max() / np.abs(ref).max()) < tol
    w.close()
    cpu.close()
    small = cuwaves.open_waves(inputs_h2o2(), precision=prec).setup()
    with pytest.raises(cuwaves.WavesError) as e:
        small.set_option(cuwaves.CUW_OPT_FFT_VARIANT, 3)
    assert e.value.code == 6
    small.close()


def inputs_h2o2():
    return systems.build_inputs(systems.water_box(2, box=10.0, lattice=(2, 1, 1), epw_psi_ry=25.0, grid=(32, 32, 32)))
