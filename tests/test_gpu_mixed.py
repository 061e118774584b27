"""The mixed-precision path (CUW_PREC_MIXED) against the FP64 path.

The contractions (<p|psi>, ADDPRO, overlaps, ADDOPSI/ADDOPROJ and the force
contraction) run as three-term tf32 products on the tcgen05 tensor cores; the
FFTs and V_loc*psi run in FP32; the orthonormality solve and the energy and
force sums stay FP64.  Both handles start from the same state and are compared
after the same operations.  Tolerances (the mixed-path targets):
  <p|psi>, H|psi>                 relative 2e-6 of max|.|
  total energy                    1e-6 Ha per atom
  forces                          1e-4 Ha/bohr
  PSI after the steps             relative 1e-4 of max|.|
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import cuwaves  # noqa: E402
from cuwaves import CUW_HPSI, CUW_PREC_FP64, CUW_PREC_MIXED, CUW_PSI0, CUW_PSIM, systems  # noqa: E402

CASES = {
    "Si8-20Ry": lambda: systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry"),
    "H2O2": lambda: systems.water_box(2, box=10.0, lattice=(2, 1, 1), epw_psi_ry=25.0, grid=(32, 32, 32)),
    "Si64": lambda: systems.named_system("Si64"),
    "Si32": lambda: systems.serving_system("Si", 32, 1),
}


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pair(name):
    inp = systems.build_inputs(CASES[name]())
    ref = cuwaves.open_waves(inp, precision=CUW_PREC_FP64).setup().initialize()
    mix = cuwaves.open_waves(inp, precision=CUW_PREC_MIXED).setup()
    for which in (CUW_PSI0, CUW_PSIM):
        mix.upload_psi(which, ref.download_psi(which))
    mix.set_proj(ref.get_proj())
    mix.set_rlam0(ref.get_rlam0())
    return inp, ref, mix


@pytest.mark.parametrize("name", ["Si8-20Ry", "H2O2", "Si64"])
def test_mixed_projections_and_hpsi(name):
    inp, ref, mix = pair(name)
    want = ref.get_proj()
    mix.projections()
    e = rel(mix.get_proj(), want)
    print(f"{name}: <p|psi> mixed vs FP64 {e:.2e}")
    assert e < 2e-6
    ref.hpsi()
    mix.hpsi()
    e = rel(mix.download_psi(CUW_HPSI), ref.download_psi(CUW_HPSI))
    print(f"{name}: H|psi> mixed vs FP64 {e:.2e}")
    assert e < 2e-6


@pytest.mark.parametrize("name", ["Si8-20Ry", "Si32", "Si64"])
def test_mixed_forces_same_state(name):
    """Forces of one state: the FP64 contraction against the tcgen05 one
    (Si8: one K chunk, per-tile kernel; Si32 and Si64: 4 and 8 chunks, the
    persistent kernel with the psi0 tile resident in tensor memory)."""
    inp, ref, mix = pair(name)
    fr, fm = ref.force(), mix.force()
    d = float(np.abs(fm - fr).max())
    print(f"{name}: forces mixed vs FP64 max |dF| {d:.2e} Ha/bohr (max |F| {np.abs(fr).max():.2e})")
    assert d < 2e-6


@pytest.mark.parametrize("name,nsteps", [("Si8-20Ry", 5), ("H2O2", 5), ("Si64", 3)])
def test_mixed_cp_steps(name, nsteps):
    """CP steps with moving atoms: energy per atom, forces, wave functions."""
    inp, ref, mix = pair(name)
    nat = inp["nat"]
    worst_e = worst_f = 0.0
    for step in range(nsteps):
        orf, frf = ref.cp_step(move_atoms=True)
        omx, fmx = mix.cp_step(move_atoms=True)
        de = abs(omx[0] - orf[0]) / nat
        df = float(np.abs(fmx - frf).max())
        worst_e, worst_f = max(worst_e, de), max(worst_f, df)
        assert de < 1e-6, f"step {step}: |dE|/atom {de:.2e}"
        assert df < 1e-4, f"step {step}: |dF| {df:.2e}"
    print(f"{name}: {nsteps} steps, max |dE|/atom {worst_e:.2e}, max |dF| {worst_f:.2e} Ha/bohr")
    e = rel(mix.download_psi(CUW_PSI0), ref.download_psi(CUW_PSI0))
    print(f"{name}: psi after {nsteps} steps, mixed vs FP64 {e:.2e}")
    assert e < 1e-4
