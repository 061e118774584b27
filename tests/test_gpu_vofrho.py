"""POTENTIAL$VOFRHO and the self-consistent CP step on the GPU, against the
oracle through the C ABI.

Tolerances (FP64):
  V(r), VQLM                       relative 1e-10 of max|.|
  EHARTREE, EXC, RHOB              1e-8 Ha (absolute)
  forces                           1e-8 Ha/bohr
  self-consistent CP steps         energies 1e-8 Ha, forces 1e-6 Ha/bohr,
                                   equal ORTHO_X iteration counts,
                                   psi relative 1e-8 after the steps
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import cuwaves  # noqa: E402
from cuwaves import CUW_OPT_SELFCONSISTENT, CUW_PREC_MIXED, CUW_PSI0, CUW_PSIM, systems  # noqa: E402

CASES = {
    "Si8": lambda: systems.named_system("Si8"),
    "H2O2": lambda: systems.water_box(2, box=10.0, lattice=(2, 1, 1), epw_psi_ry=25.0, grid=(32, 32, 32)),
    "Si64": lambda: systems.named_system("Si64"),
}


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def sync_state(src, dst):
    dst.upload_psi(CUW_PSI0, src.download_psi(CUW_PSI0))
    dst.upload_psi(CUW_PSIM, src.download_psi(CUW_PSIM))
    dst.set_proj(src.get_proj())
    dst.set_rlam0(src.get_rlam0())


def pair(name, oracle, precision=cuwaves.CUW_PREC_FP64):
    inp = systems.build_inputs(CASES[name]())
    gpu = cuwaves.open_waves(inp, precision=precision).setup().initialize().set_rhoset()
    cpu = oracle.open_oracle(inp).setup().set_rhoset()
    sync_state(gpu, cpu)
    return inp, gpu, cpu


@pytest.mark.parametrize("name", ["Si8", "H2O2", "Si64"])
def test_vofrho_matches_oracle(name, oracle):
    """V(r), energies, forces and VQLM from the same density; then from the
    density of PSI0 formed on each side."""
    inp, gpu, cpu = pair(name, oracle)
    rho = cpu.density()
    vg, eg, fg, qg = gpu.vofrho(rho)
    vc, ec, fc, qc = cpu.vofrho(rho)
    assert rel(vg, vc) < 1e-10
    for k in ("ehartree", "exc", "rhob"):
        assert abs(eg[k] - ec[k]) < 1e-8, (k, eg[k], ec[k])
    assert np.abs(fg - fc).max() < 1e-8
    assert rel(qg, qc) < 1e-10
    vg2, eg2, fg2, _ = gpu.vofrho()
    vc2, ec2, fc2, _ = cpu.vofrho()
    assert rel(vg2, vc2) < 1e-10
    assert abs(eg2["ehartree"] - ec2["ehartree"]) < 1e-8 and abs(eg2["exc"] - ec2["exc"]) < 1e-8
    assert np.abs(fg2 - fc2).max() < 1e-8
    # the potential became the handle's: H|psi> with it agrees too
    gpu.hpsi()
    cpu.hpsi()
    assert rel(gpu.download_psi(cuwaves.CUW_HPSI), cpu.download_psi(cuwaves.CUW_HPSI)) < 1e-10


def test_vofrho_mixed_handle(oracle):
    """On a mixed-precision handle the potential is still formed in FP64."""
    inp, gpu, cpu = pair("Si8", oracle, precision=CUW_PREC_MIXED)
    rho = cpu.density()
    vg, eg, fg, _ = gpu.vofrho(rho)
    vc, ec, fc, _ = cpu.vofrho(rho)
    assert rel(vg, vc) < 1e-10
    assert abs(eg["exc"] - ec["exc"]) < 1e-8
    assert np.abs(fg - fc).max() < 1e-8


@pytest.mark.parametrize("name,nsteps,move", [("Si8", 6, True), ("H2O2", 4, True)])
def test_selfconsistent_cp_steps(name, nsteps, move, oracle):
    """CP steps with V(r) formed from the density every step (replayed as CUDA
    graphs after the first steps) against the oracle step by step."""
    inp, gpu, cpu = pair(name, oracle)
    for w in (gpu, cpu):
        w.set_option(CUW_OPT_SELFCONSISTENT, 1)
    for step in range(nsteps):
        og, fg = gpu.cp_step(move_atoms=move)
        oc, fc = cpu.cp_step(move_atoms=move)
        assert og[4] == oc[4], f"step {step}: ortho iterations {og[4]} vs {oc[4]}"
        for k in (0, 1, 2, 3, 5, 6, 7):
            assert abs(og[k] - oc[k]) < 1e-8 * max(1.0, abs(oc[k]) / 100), f"step {step}: out[{k}] {og[k]} vs {oc[k]}"
        assert np.abs(fg - fc).max() < 1e-6, f"step {step}: forces"
    assert rel(gpu.download_psi(CUW_PSI0), cpu.download_psi(CUW_PSI0)) < 1e-8
    assert gpu.graph_stats()[1] > 0  # later steps were graph replays
    # switched off again: V stays as the last step left it
    gpu.set_option(CUW_OPT_SELFCONSISTENT, 0)
    cpu.set_option(CUW_OPT_SELFCONSISTENT, 0)
    og, _ = gpu.cp_step(move_atoms=move)
    oc, _ = cpu.cp_step(move_atoms=move)
    assert abs(og[0] - oc[0]) < 1e-8 * max(1.0, abs(oc[0]) / 100) and og[5] == 0.0
