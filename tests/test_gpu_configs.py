"""The benchmark configurations themselves, on the GPU.

- Si8 exactly as the CPU-runnable configuration: a = 10.26 bohr, 16 bands,
  30/60 Ry, 32^3 grid, 10 FP64 CP steps against the oracle step by step.
- The reference-rule grids (BOXSPH + LIB$FFTADJUSTGRD for the density cutoff:
  28^3 for Si8 and 56^3 for Si64), which the C ABI takes like any other grid,
  against the oracle at the FP64 tolerances.
- The precision configuration, 32 H2O molecules at 40/80 Ry on 72^3, mixed
  precision against the FP64 path from the same state.
Every step is also checked with the orthonormality test of
WAVES$ORTHOGONALIZE (src/paw_waves2.f90:421-460, cuwaves_overlap_check).
Tolerances as in test_gpu_parity (FP64) and test_gpu_mixed (mixed path).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import cuwaves  # noqa: E402
from cuwaves import CUW_PREC_FP64, CUW_PREC_MIXED, CUW_PSI0, CUW_PSIM, systems  # noqa: E402


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def sync_state(src, dst):
    dst.upload_psi(CUW_PSI0, src.download_psi(CUW_PSI0))
    dst.upload_psi(CUW_PSIM, src.download_psi(CUW_PSIM))
    dst.set_proj(src.get_proj())
    dst.set_rlam0(src.get_rlam0())


def run_pair(name, inp, oracle, nsteps, move):
    gpu = cuwaves.open_waves(inp).setup().initialize()
    cpu = oracle.open_oracle(inp).setup()
    sync_state(gpu, cpu)
    mg, dg = gpu.overlap_check()
    mc, dc = cpu.overlap_check()
    assert np.abs(mg - mc).max() < 1e-10, f"{name}: overlap matrices differ"
    for step in range(nsteps):
        og, fg = gpu.cp_step(move_atoms=move)
        oc, fc = cpu.cp_step(move_atoms=move)
        assert og[4] == oc[4], f"{name} step {step}: ortho iterations {og[4]} vs {oc[4]}"
        tol = 1e-8 * max(1.0, abs(oc[0]) / 100)
        assert abs(og[0] - oc[0]) < tol, f"{name} step {step}: E {og[0]} vs {oc[0]}"
        for k in (1, 2, 3):
            assert abs(og[k] - oc[k]) < tol, f"{name} step {step}: out[{k}] {og[k]} vs {oc[k]}"
        assert np.abs(fg - fc).max() < 1e-6, f"{name} step {step}: forces"
        _, dg = gpu.overlap_check()
        _, dc = cpu.overlap_check()
        # the ORTHO_X loop stops at max|<psi|O|psi> - 1| < 1e-8
        assert dg < 1e-7 and dc < 1e-7, f"{name} step {step}: orthonormality {dg:.2e} / {dc:.2e}"
    assert rel(gpu.download_psi(CUW_PSI0), cpu.download_psi(CUW_PSI0)) < 1e-8
    gpu.close()
    cpu.close()


def test_config_si8_ten_steps(oracle):
    """The CPU-runnable configuration exactly: Si8, 16 bands, 30/60 Ry, 32^3,
    dt = 10, m = 1000, 10 FP64 CP steps."""
    inp = systems.build_inputs(systems.named_system("Si8"))
    assert inp["grid"] == (32, 32, 32) and inp["nb"] == 16
    assert inp["delt"] == 10.0 and inp["emass"] == 1000.0
    run_pair("Si8", inp, oracle, 10, False)


@pytest.mark.parametrize("name,nsteps", [("Si8-ref", 4), ("Si64-ref", 2)])
def test_reference_rule_grids(name, nsteps, oracle):
    """28^3 (Si8) and 56^3 (Si64): the grids the reference's own rule picks for
    the 60 Ry density cutoff."""
    inp = systems.build_inputs(systems.named_system(name))
    want = (28, 28, 28) if name == "Si8-ref" else (56, 56, 56)
    assert inp["grid"] == want
    run_pair(name, inp, oracle, nsteps, True)


def test_config_h2o32_mixed_vs_fp64():
    """32 H2O at 40/80 Ry on 72^3 (the precision configuration): the mixed path
    against the FP64 path over 3 CP steps with moving atoms from one state;
    energy per atom, forces, wave functions and the orthonormality residual."""
    inp = systems.build_inputs(systems.named_system("H2O32"))
    assert inp["grid"] == (72, 72, 72)
    ref = cuwaves.open_waves(inp, precision=CUW_PREC_FP64).setup().initialize()
    mix = cuwaves.open_waves(inp, precision=CUW_PREC_MIXED).setup()
    sync_state(ref, mix)
    nat = inp["nat"]
    for step in range(3):
        orf, frf = ref.cp_step(move_atoms=True)
        omx, fmx = mix.cp_step(move_atoms=True)
        de = abs(omx[0] - orf[0]) / nat
        df = float(np.abs(fmx - frf).max())
        assert de < 1e-6, f"step {step}: |dE|/atom {de:.2e}"
        assert df < 1e-4, f"step {step}: |dF| {df:.2e}"
        _, dr = ref.overlap_check()
        _, dm = mix.overlap_check()
        print(f"H2O32 step {step}: |dE|/atom {de:.2e}, |dF| {df:.2e}, orthonormality FP64 {dr:.2e} mixed {dm:.2e}")
        assert dr < 1e-7
        assert dm < 1e-4  # the reference's own bound (src/paw_waves2.f90:456)
    assert rel(mix.download_psi(CUW_PSI0), ref.download_psi(CUW_PSI0)) < 1e-4
