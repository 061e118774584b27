"""Parity of the CUDA engine with the CPU oracle, through the C ABI.

Each test puts the engine and the oracle into the same state (same seeded
inputs, the same orthonormal PSI0/PSIM, PROJ and RLAM0), runs one WAVES
operation on both and compares.  Tolerances (FP64 path):
  H|psi>, PSI after a step       relative 1e-10 / 1e-9 of max|.|
  energies                       1e-8 Ha absolute
  forces                         1e-6 Ha/bohr absolute
  PROJ, overlaps                 relative 1e-10
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import cuwaves  # noqa: E402
from cuwaves import CUW_HPSI, CUW_OPSI, CUW_PSI0, CUW_PSIM, WavesError, systems  # noqa: E402

CASES = {
    "Si8-20Ry": lambda: systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry"),
    "Si8": lambda: systems.named_system("Si8"),
    "Si2mol": lambda: systems.molecule_box("Si2", box=12.0, epw_psi_ry=15.0, grid=(20, 20, 20)),
    "H2O2": lambda: systems.water_box(2, box=10.0, lattice=(2, 1, 1), epw_psi_ry=25.0, grid=(32, 32, 32)),
    "Si6": lambda: systems.si_small(6, epw_psi_ry=15.0, grid=(20, 20, 20)),
}


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def inputs_cache():
    return {}


def make_pair(name, oracle, cache):
    if name not in cache:
        cache[name] = systems.build_inputs(CASES[name]())
    inp = cache[name]
    gpu = cuwaves.open_waves(inp).setup().initialize()
    cpu = oracle.open_oracle(inp).setup()
    sync_state(gpu, cpu)
    return inp, gpu, cpu


def sync_state(src, dst):
    """Copy PSI0, PSIM, PROJ and RLAM0 from src to dst."""
    dst.upload_psi(CUW_PSI0, src.download_psi(CUW_PSI0))
    dst.upload_psi(CUW_PSIM, src.download_psi(CUW_PSIM))
    dst.set_proj(src.get_proj())
    dst.set_rlam0(src.get_rlam0())


@pytest.mark.parametrize("name", ["Si8-20Ry"])
def test_roundtrip_bits(name, oracle, inputs_cache):
    inp, gpu, _ = make_pair(name, oracle, inputs_cache)
    rng = np.random.default_rng(5)
    x = rng.normal(size=(inp["nbh"], inp["ngl"])) + 1j * rng.normal(size=(inp["nbh"], inp["ngl"]))
    for which in (CUW_PSI0, CUW_PSIM, CUW_HPSI, CUW_OPSI):
        gpu.upload_psi(which, x)
        assert np.array_equal(gpu.download_psi(which), x)
    p = rng.normal(size=(gpu.npro, inp["nbh"])) + 1j * rng.normal(size=(gpu.npro, inp["nbh"]))
    gpu.set_proj(p)
    assert np.array_equal(gpu.get_proj(), p)
    r = rng.normal(size=(inp["nb"], inp["nb"])) + 0j
    gpu.set_rlam0(r)
    assert np.array_equal(gpu.get_rlam0(), r)


@pytest.mark.parametrize("name", ["Si8-20Ry", "H2O2", "Si6"])
def test_fft_identity(name, oracle, inputs_cache):
    """With V=1 and DH=0, H|psi> = psi + 1/2 G^2 psi: the FFT pair is an identity."""
    inp, gpu, _ = make_pair(name, oracle, inputs_cache)
    gpu.set_potential(np.ones_like(inp["v"]))
    gpu.set_dh(np.zeros_like(inp["dh"]))
    gpu.hpsi()
    psi = gpu.download_psi(CUW_PSI0)
    want = psi * (1.0 + 0.5 * inp["g2"][None, :])
    assert rel(gpu.download_psi(CUW_HPSI), want) < 1e-12


@pytest.mark.parametrize("name", ["Si8-20Ry", "Si8", "H2O2", "Si2mol", "Si6"])
def test_projections(name, oracle, inputs_cache):
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    gpu.projections()
    cpu.projections()
    assert rel(gpu.get_proj(), cpu.get_proj()) < 1e-10


@pytest.mark.parametrize("name", ["Si8-20Ry", "Si8", "H2O2", "Si2mol", "Si6"])
def test_hpsi(name, oracle, inputs_cache):
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    gpu.hpsi()
    cpu.hpsi()
    assert rel(gpu.download_psi(CUW_HPSI), cpu.download_psi(CUW_HPSI)) < 1e-10


@pytest.mark.parametrize("name", ["Si8", "H2O2"])
def test_energies(name, oracle, inputs_cache):
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    # give PSIM a different value so that the fictitious kinetic energy is nonzero
    rng = np.random.default_rng(7)
    pm = gpu.download_psi(CUW_PSI0) * (1 + 1e-3 * rng.normal(size=(inp["nbh"], inp["ngl"])))
    gpu.upload_psi(CUW_PSIM, pm)
    cpu.upload_psi(CUW_PSIM, pm)
    assert abs(gpu.ekin() - cpu.ekin()) < 1e-8
    eg, vg = gpu.wavekinetic()
    ec, vc = cpu.wavekinetic()
    assert abs(eg - ec) < 1e-8 * max(1.0, abs(ec))
    assert np.abs(vg - vc).max() < 1e-8 * max(1.0, np.abs(vc).max())
    gpu.hpsi()
    cpu.hpsi()
    assert np.abs(gpu.expectation() - cpu.expectation()).max() < 1e-8


def test_energies_unequal_occupations(oracle, inputs_cache):
    """Occupations that differ inside a super wave function exercise the
    PSI(-G) terms of WAVES_EKIN and WAVES_WAVEKINETIC."""
    inp, gpu, cpu = make_pair("Si8-20Ry", oracle, inputs_cache)
    occ = inp["occ"].copy()
    occ[-3:] = [1.0, 0.5, 0.0]
    gpu.set_occ(occ)
    cpu.set_occ(occ)
    rng = np.random.default_rng(8)
    pm = gpu.download_psi(CUW_PSI0) * (1 + 1e-3 * rng.normal(size=(inp["nbh"], inp["ngl"])))
    gpu.upload_psi(CUW_PSIM, pm)
    cpu.upload_psi(CUW_PSIM, pm)
    assert abs(gpu.ekin() - cpu.ekin()) < 1e-8
    assert abs(gpu.wavekinetic()[0] - cpu.wavekinetic()[0]) < 1e-8
    assert np.abs(gpu.force() - cpu.force()).max() < 1e-6


@pytest.mark.parametrize("name", ["Si8-20Ry", "Si8", "H2O2", "Si6"])
def test_force(name, oracle, inputs_cache):
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    rng = np.random.default_rng(9)
    lam = rng.normal(size=(inp["nb"], inp["nb"])) * 0.1
    lam = (lam + lam.T) + 0j
    gpu.set_rlam0(lam)
    cpu.set_rlam0(lam)
    fg, fc = gpu.force(), cpu.force()
    assert np.abs(fg - fc).max() < 1e-6
    assert np.abs(fg - fc).max() < 1e-9 * max(1.0, np.abs(fc).max())


@pytest.mark.parametrize("name", ["Si8-20Ry", "Si8", "H2O2", "Si6", "Si2mol"])
def test_density_and_denmat(name, oracle, inputs_cache):
    """WAVES_DENSITY (pseudo density on the grid) and WAVES$DENMAT (one-centre
    and energy-weighted density matrices) against the oracle, FP64 path, with a
    nonzero Lagrange history so that EDENMAT is not trivial; unequal
    occupations exercise the s2 terms of the super wave functions."""
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    rng = np.random.default_rng(11)
    nb = inp["nb"]
    lam = rng.normal(size=(nb, nb)) * 0.1 + 1j * rng.normal(size=(nb, nb)) * 0.01
    occ = np.array(inp["occ"], dtype=np.float64)
    occ[-1] = 0.5
    for w in (gpu, cpu):
        w.set_rlam0(lam)
        w.set_occ(occ)
    rg, rc = gpu.density(), cpu.density()
    assert rel(rg, rc) < 1e-12
    (dg, eg), (dc, ec) = gpu.denmat(), cpu.denmat()
    assert rel(dg, dc) < 1e-12 and rel(eg, ec) < 1e-12
    assert np.abs(dg.imag).max() == 0.0


def test_density_mixed_path(oracle, inputs_cache):
    """The density on the mixed path (FP32 G->R transforms, FP64 sums)."""
    name = "Si8-20Ry"
    if name not in inputs_cache:
        inputs_cache[name] = systems.build_inputs(CASES[name]())
    inp = inputs_cache[name]
    mix = cuwaves.open_waves(inp, precision=cuwaves.CUW_PREC_MIXED).setup().initialize()
    cpu = oracle.open_oracle(inp).setup()
    sync_state(mix, cpu)
    assert rel(mix.density(), cpu.density()) < 2e-6
    (dg, _), (dc, _) = mix.denmat(), cpu.denmat()
    assert rel(dg, dc) < 1e-12  # PROJ is the same state; the sums are FP64 on both paths


@pytest.mark.parametrize("name", ["Si8-20Ry", "H2O2"])
def test_propagate(name, oracle, inputs_cache):
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    gpu.hpsi()
    cpu.hpsi()
    gpu.propagate()
    cpu.propagate()
    assert rel(gpu.download_psi(CUW_PSIM), cpu.download_psi(CUW_PSIM)) < 1e-10
    with pytest.raises(WavesError) as e:
        gpu.propagate()  # HPSI consumed: the reference stops here too
    assert e.value.code == 3


@pytest.mark.parametrize("name", ["Si8-20Ry", "Si8", "H2O2", "Si6"])
def test_orthogonalize(name, oracle, inputs_cache):
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    for w in (gpu, cpu):
        w.hpsi()
        w.propagate()
    sync_state(gpu, cpu)
    ig = gpu.orthogonalize()
    ic = cpu.orthogonalize()
    assert ig == ic
    assert rel(gpu.download_psi(CUW_PSIM), cpu.download_psi(CUW_PSIM)) < 1e-9
    assert rel(gpu.get_proj(), cpu.get_proj()) < 1e-9
    assert np.abs(gpu.get_rlam0() - cpu.get_rlam0()).max() < 1e-8


@pytest.mark.parametrize("name", ["Si8", "H2O2"])
def test_lyapunov_tolerance(name, oracle, inputs_cache):
    """The inner Lyapunov solve of ORTHO_X at its default accuracy (1e-2 while
    the residual is far from EPS, 1e-5 in the last iterations) against the
    solve to rounding (CUW_OPT_LYAP_TOL = 0), from one state over six CP steps
    with moving atoms: the same ORTHO_X iteration counts, energies within
    1e-9 Ha and forces within 1e-8 Ha/bohr, with fewer fixed-point sweeps."""
    inp, ref, cpu = make_pair(name, oracle, inputs_cache)
    cpu.close()
    ref.set_option(cuwaves.CUW_OPT_LYAP_TOL, 0.0)
    w = cuwaves.open_waves(inp).setup()
    sync_state(ref, w)
    s0 = (ref.ortho_stats()["fixed_point_sweeps"], w.ortho_stats()["fixed_point_sweeps"])
    for step in range(6):
        (oa, fa), (ob, fb) = ref.cp_step(move_atoms=True), w.cp_step(move_atoms=True)
        assert oa[4] == ob[4], f"step {step}: iterations {oa[4]} vs {ob[4]}"
        assert abs(oa[0] - ob[0]) < 1e-9 and np.abs(fa - fb).max() < 1e-8
    s1 = (ref.ortho_stats()["fixed_point_sweeps"], w.ortho_stats()["fixed_point_sweeps"])
    assert s1[1] - s0[1] < s1[0] - s0[0]
    ref.close()
    w.close()


def test_gramschmidt(oracle, inputs_cache):
    inp = systems.build_inputs(CASES["Si8-20Ry"]())
    gpu = cuwaves.open_waves(inp).setup()
    cpu = oracle.open_oracle(inp).setup()
    for w in (gpu, cpu):
        w.gramschmidt(CUW_PSI0, inp["r0"])
    assert rel(gpu.download_psi(CUW_PSI0), cpu.download_psi(CUW_PSI0)) < 1e-10


def test_large_band_count(oracle):
    """NB = 256, beyond one CTA's shared memory: the cluster Gram-Schmidt, the
    cluster Jacobi eigensolver of the first ORTHO_X call and the ORTHO_X
    cluster kernel for NB > 128, against the oracle (Gram-Schmidt, then two
    CP steps with moving atoms)."""
    inp = systems.build_inputs(systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, nb=256, name="Si8-nb256"))
    assert inp["nb"] == 256
    gpu = cuwaves.open_waves(inp).setup()
    cpu = oracle.open_oracle(inp).setup()
    for which in (CUW_PSI0, CUW_PSIM):
        for w in (gpu, cpu):
            w.gramschmidt(which, inp["r0"])
        # 256 sequential orthogonalisation steps from random vectors: the
        # rounding of the two machines accumulates to a few 1e-10
        assert rel(gpu.download_psi(which), cpu.download_psi(which)) < 1e-9
    gpu.projections()
    cpu.projections()
    sync_state(gpu, cpu)
    for step in range(2):
        og, fg = gpu.cp_step(move_atoms=True)
        oc, fc = cpu.cp_step(move_atoms=True)
        assert og[4] == oc[4], f"step {step}: ortho iterations {og[4]} vs {oc[4]}"
        tol = 1e-8 * max(1.0, abs(oc[0]) / 100)
        assert abs(og[0] - oc[0]) < tol, f"step {step}: E {og[0]} vs {oc[0]}"
        assert np.abs(fg - fc).max() < 1e-6
    assert gpu.ortho_stats()["eigendecompositions"] >= 1
    assert rel(gpu.download_psi(CUW_PSI0), cpu.download_psi(CUW_PSI0)) < 1e-8
    gpu.close()
    cpu.close()


@pytest.mark.parametrize("name,nsteps,move", [("Si8-20Ry", 8, False), ("Si8", 5, True), ("H2O2", 5, True)])
def test_cp_steps(name, nsteps, move, oracle, inputs_cache):
    """Full CP steps (TIMESTEP order) on both engines, compared step by step."""
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    for step in range(nsteps):
        og, fg = gpu.cp_step(move_atoms=move)
        oc, fc = cpu.cp_step(move_atoms=move)
        assert og[4] == oc[4], f"step {step}: ortho iterations {og[4]} vs {oc[4]}"
        assert abs(og[0] - oc[0]) < 1e-8, f"step {step}: E {og[0]} vs {oc[0]}"
        assert abs(og[1] - oc[1]) < 1e-8
        assert abs(og[2] - oc[2]) < 1e-8
        assert abs(og[3] - oc[3]) < 1e-8
        assert np.abs(fg - fc).max() < 1e-6
    assert rel(gpu.download_psi(CUW_PSI0), cpu.download_psi(CUW_PSI0)) < 1e-8


@pytest.mark.parametrize("name,swap", [("Si8", 0), ("Si8", 1), ("H2O2", 1)])
def test_cp_steps_safeortho_false(name, swap, oracle, inputs_cache):
    """SAFEORTHO = F (src/paw_waves2.f90:306-386): inside the CP step the
    cluster kernel of WAVES_ORTHO_Y_C replaces ORTHO_X, with the states in the
    order of the RLAM0 diagonal when SWAPSTATES = T (the warp-scan exchange
    sort); step by step against the oracle, from a state whose RLAM0 came from
    ordinary steps."""
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    for w in (gpu, cpu):
        w.cp_step(move_atoms=True)
    sync_state(gpu, cpu)
    d = np.diag(gpu.get_rlam0()).real
    if swap:
        assert not np.all(np.diff(d) >= 0)  # the order changes
    for w in (gpu, cpu):
        w.set_option(cuwaves.CUW_OPT_SWAPSTATES, swap)
        w.set_option(cuwaves.CUW_OPT_SAFEORTHO, 0)
    for step in range(4):
        og, fg = gpu.cp_step(move_atoms=True)
        oc, fc = cpu.cp_step(move_atoms=True)
        assert og[4] == 0 and oc[4] == 0
        for k in range(4):
            assert abs(og[k] - oc[k]) < 1e-8, f"step {step}: out[{k}] {og[k]} vs {oc[k]}"
        assert np.abs(fg - fc).max() < 1e-6
    assert rel(gpu.download_psi(CUW_PSI0), cpu.download_psi(CUW_PSI0)) < 1e-8
    assert np.abs(gpu.get_rlam0() - cpu.get_rlam0()).max() < 1e-8
    gpu.close()
    cpu.close()


def _cell_friction(inp):
    """PSIANNEMAT is the cell's strain rate times DELT/2: with entries of 2e-5
    and EMASS*EMASSCG2 near 130, ANNEEVEC stays within a few 1e-2 of ANNEE
    over the sphere."""
    rng = np.random.default_rng(9)
    return dict(fricmat=rng.normal(size=(3, 3)) * 2e-5, emass=inp["emass"], emasscg2=inp["emasscg2"],
                dbucket=rng.uniform(0.0, 0.2, size=inp["ngl"]))


@pytest.mark.parametrize("name", ["Si8-20Ry", "H2O2"])
def test_propagate_cell_friction(name, oracle, inputs_cache):
    """WAVES$PROPAGATE with the G-dependent friction of a moving cell
    (ANNEEVEC of WAVES_DMPSI, src/paw_waves1.f90:6524-6543, 6676-6711): the
    standalone propagation and CP steps (the propagation fused into the
    back-projection) against the oracle."""
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    fr = _cell_friction(inp)
    for w in (gpu, cpu):
        w.set_dynamics(inp["delt"], 0.02)
        w.set_cell_friction(**fr)
        w.hpsi()
        w.propagate()
    assert rel(gpu.download_psi(CUW_PSIM), cpu.download_psi(CUW_PSIM)) < 1e-10
    gpu.close()
    cpu.close()
    # CP steps from an orthonormal state (PSIM above is the unconstrained psi(+))
    inp, gpu, cpu = make_pair(name, oracle, inputs_cache)
    for w in (gpu, cpu):
        w.set_dynamics(inp["delt"], 0.02)
        w.set_cell_friction(**fr)
    for step in range(3):
        og, fg = gpu.cp_step(move_atoms=True)
        oc, fc = cpu.cp_step(move_atoms=True)
        assert og[4] == oc[4]
        for k in range(4):
            assert abs(og[k] - oc[k]) < 1e-8, f"step {step}: out[{k}] {og[k]} vs {oc[k]}"
        assert np.abs(fg - fc).max() < 1e-6
    assert rel(gpu.download_psi(CUW_PSI0), cpu.download_psi(CUW_PSI0)) < 1e-8
    gpu.close()
    cpu.close()


def test_cell_friction_mixed_path(oracle, inputs_cache):
    """The friction in the tcgen05 back-projection epilogue of the mixed path:
    one CP step agrees with the FP64 path under the same friction to the mixed
    path's precision, and differs from a step without it."""
    inp = systems.build_inputs(CASES["Si8"]())
    fr = _cell_friction(inp)
    res = {}
    for prec, fric in ((cuwaves.CUW_PREC_FP64, True), (cuwaves.CUW_PREC_MIXED, True), (cuwaves.CUW_PREC_MIXED, False)):
        w = cuwaves.open_waves(inp, precision=prec).setup().initialize()
        w.set_dynamics(inp["delt"], 0.02)
        if fric:
            w.set_cell_friction(**fr)
        w.cp_step(move_atoms=False)
        res[(prec, fric)] = w.download_psi(CUW_PSI0)
        w.close()
    a, b = res[(cuwaves.CUW_PREC_FP64, True)], res[(cuwaves.CUW_PREC_MIXED, True)]
    c = res[(cuwaves.CUW_PREC_MIXED, False)]
    assert rel(b, a) < 1e-5
    assert rel(c, a) > 10 * rel(b, a)


def test_not_converged_status_and_recovery(oracle, inputs_cache):
    """A forced non-convergence (max_iter=1) is reported as a status and the
    handle stays usable (the reference stops the run instead)."""
    inp, gpu, cpu = make_pair("Si8-20Ry", oracle, inputs_cache)
    gpu.hpsi()
    gpu.propagate()
    with pytest.raises(WavesError) as e:
        gpu.orthogonalize(max_iter=1, eps=1e-14)
    assert e.value.code == 4
    # the context is still usable: a fresh step works
    gpu2 = cuwaves.open_waves(inp).setup().initialize()
    out, _ = gpu2.cp_step()
    assert np.isfinite(out[0])


def test_nan_input_detected(oracle, inputs_cache):
    """A NaN planted in the host input is reported, not propagated silently."""
    inp = systems.build_inputs(CASES["Si8-20Ry"]())
    gpu = cuwaves.open_waves(inp).setup()
    psi = inp["psi"].copy()
    psi[0, 3] = np.nan
    gpu.upload_psi(CUW_PSI0, psi)
    with pytest.raises(WavesError) as e:
        gpu.gramschmidt(CUW_PSI0, inp["r0"])
    assert e.value.code == 7
    gpu2 = cuwaves.open_waves(inp).setup().initialize()
    assert np.isfinite(gpu2.ekin())


@pytest.mark.parametrize("name", ["Si64", "H2O32"])
def test_full_size_step(name, oracle):
    """The benchmark systems at full size (64^3 and 72^3 grids): H|psi> and one
    complete CP step against the oracle."""
    inp = systems.build_inputs(systems.named_system(name))
    gpu = cuwaves.open_waves(inp).setup().initialize()
    cpu = oracle.open_oracle(inp).setup()
    sync_state(gpu, cpu)
    gpu.hpsi()
    cpu.hpsi()
    assert rel(gpu.download_psi(CUW_HPSI), cpu.download_psi(CUW_HPSI)) < 1e-10
    og, fg = gpu.cp_step(move_atoms=True)
    oc, fc = cpu.cp_step(move_atoms=True)
    assert og[4] == oc[4]
    assert abs(og[0] - oc[0]) < 1e-8 * max(1.0, abs(oc[0]) / 100)
    assert np.abs(fg - fc).max() < 1e-6
    assert rel(gpu.download_psi(CUW_PSI0), cpu.download_psi(CUW_PSI0)) < 1e-9


@pytest.mark.parametrize("precision", [cuwaves.CUW_PREC_FP64, cuwaves.CUW_PREC_MIXED])
def test_restart_records(precision, oracle, inputs_cache, tmp_path):
    """WAVES$WRITE / WAVES$READ on the device: the engine reads the oracle's
    file bit for bit, writes back the same bytes, maps a file whose G vectors
    are permuted and partly missing, and continues the run like the oracle."""
    import restart_file as rf

    name = "Si8-20Ry"
    if name not in inputs_cache:
        inputs_cache[name] = systems.build_inputs(CASES[name]())
    inp = inputs_cache[name]
    cpu = oracle.open_oracle(inp).setup().initialize()
    for _ in range(3):
        cpu.cp_step()
    a = tmp_path / "cpu.rst"
    cpu.write_restart(a, inp["rbas"])
    gpu = cuwaves.open_waves(inp, precision=precision).setup()
    gpu.read_restart(a)
    assert np.array_equal(gpu.download_psi(CUW_PSI0), cpu.download_psi(CUW_PSI0))
    assert np.array_equal(gpu.download_psi(CUW_PSIM), cpu.download_psi(CUW_PSIM))
    assert np.array_equal(gpu.get_rlam0(), cpu.get_rlam0())
    b = tmp_path / "gpu.rst"
    gpu.write_restart(b, inp["rbas"])
    assert b.read_bytes() == a.read_bytes()
    # RBAS from the handle's GBAS
    gpu.write_restart(tmp_path / "g2.rst")
    r = rf.parse_waves(rf.read_records(tmp_path / "g2.rst"))["rbas"]
    assert np.abs(r - np.asarray(inp["rbas"])).max() < 1e-12 * np.abs(inp["rbas"]).max()

    # the run continues from the file (PROJ formed from PSI0 on both sides)
    gpu.projections()
    cpu.projections()
    for _ in range(2):
        (og, fg), (oc, fc) = gpu.cp_step(), cpu.cp_step()
    tol_e = 1e-8 if precision == cuwaves.CUW_PREC_FP64 else 1e-6 * inp["nat"]
    tol_f = 1e-6 if precision == cuwaves.CUW_PREC_FP64 else 1e-4
    assert abs(og[0] - oc[0]) < tol_e
    assert np.abs(fg - fc).max() < tol_f

    # permuted and truncated G vectors: mapped by G vector, the rest zero
    d = rf.parse_waves(rf.read_records(a))
    perm = np.random.default_rng(3).permutation(d["ngg"])
    keep = d["ngg"] - 40
    c = tmp_path / "perm.rst"
    rf.write_records(c, rf.permuted(rf.read_records(a), perm, keep))
    gpu.read_restart(c)
    want = d["psi"][0].copy()
    want[:, perm[keep:]] = 0.0
    assert np.array_equal(gpu.download_psi(CUW_PSI0), want)
    # a static restart (NWAVE = 1) starts PSIM from PSI0
    rf.write_records(tmp_path / "static.rst", rf.static(rf.read_records(a)))
    gpu.read_restart(tmp_path / "static.rst")
    assert np.array_equal(gpu.download_psi(CUW_PSI0), d["psi"][0])
    assert np.array_equal(gpu.download_psi(CUW_PSIM), d["psi"][0])
    # a file for another band count is refused and leaves the handle usable
    import struct
    bad = rf.read_records(a)
    bad[2] = bad[2][:16] + struct.pack("<i", inp["nb"] + 2) + bad[2][20:]
    rf.write_records(tmp_path / "bad.rst", bad)
    with pytest.raises(WavesError):
        gpu.read_restart(tmp_path / "bad.rst")
    gpu.read_restart(a)
    assert np.array_equal(gpu.download_psi(CUW_PSI0), d["psi"][0])
    # a negative G-vector count or a 2 GB record marker is an argument error
    # of the call, and the handle keeps its state
    for fname, raw in rf.damaged(a):
        (tmp_path / fname).write_bytes(raw)
        with pytest.raises(WavesError):
            gpu.read_restart(tmp_path / fname)
        assert np.array_equal(gpu.download_psi(CUW_PSI0), d["psi"][0])
