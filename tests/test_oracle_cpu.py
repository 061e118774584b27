"""CPU checks of the oracle and of the host-side index rules (no GPU).

- the MSLNG random-number known answer of the reference
  (src/paw_generalpurpose.f90:2236-2239: seed 1043618065 after 10000 draws);
- G-set ordering, MINUSG and grid rules: numpy restatement == C restatement;
- the oracle's FFT against numpy, its eigensolver against scipy;
- physical invariants of the oracle's CP dynamics (orthonormality after
  WAVES$ORTHOGONALIZE, energy conservation of order dt^2);
- regression against the committed golden fixtures.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from cuwaves import systems

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_mslng_known_answer(oracle):
    lib = oracle.library()
    seed = C.c_int(1)
    for _ in range(10000):
        lib.orc_mslng(C.byref(seed))
    assert seed.value == 1043618065


@pytest.mark.parametrize("name", ["Si8", "Si64", "H2O32"])
def test_gset_numpy_equals_oracle(name, oracle):
    s = systems.named_system(name)
    gbas, _ = systems.gbass(s.rbas)
    ig = systems.get_ig(gbas, s.epw_psi)
    lib = oracle.library()
    gb = np.asfortranarray(gbas)
    n = C.c_int()
    dp = C.POINTER(C.c_double)
    lib.orc_getig(gb.ctypes.data_as(dp), C.c_double(s.epw_psi), C.byref(n), None)
    out = np.zeros((n.value, 3), dtype=np.int32)
    lib.orc_getig(gb.ctypes.data_as(dp), C.c_double(s.epw_psi), C.byref(n), out.ctypes.data_as(C.POINTER(C.c_int)))
    assert np.array_equal(out, ig)
    mg = np.zeros(n.value, dtype=np.int32)
    assert lib.orc_minusg(n.value, out.ctypes.data_as(C.POINTER(C.c_int)), mg.ctypes.data_as(C.POINTER(C.c_int))) == 0
    assert np.array_equal(mg, systems.minus_g(ig))


def test_ngl_and_reference_grids():
    """NGL and the reference-rule grids of the benchmark systems."""
    for name, ngl, grid in [("Si8", 2945, (28, 28, 28)), ("Si64", 23847, (56, 56, 56)), ("H2O32", 27633, (56, 56, 56))]:
        s = systems.named_system(name)
        gbas, _ = systems.gbass(s.rbas)
        assert len(systems.get_ig(gbas, s.epw_psi)) == ngl
        assert systems.reference_grid(s.rbas, 2 * s.epw_psi) == grid


def test_fftadjustgrd(oracle):
    lib = oracle.library()
    for n in [1, 2, 7, 13, 27, 28, 49, 55, 57, 97, 100, 129]:
        assert lib.orc_fftadjustgrd(n) == systems.fft_adjust_grid(n)


@pytest.mark.parametrize("n", [16, 24, 28, 32, 40, 45, 56, 64, 72, 88, 96])
def test_fft1d_against_numpy(n, oracle):
    lib = oracle.library()
    rng = np.random.default_rng(n)
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    for d in (+1, -1):
        y = x.copy()
        lib.orc_fft1d(n, d, y.ctypes.data_as(C.POINTER(C.c_double)))
        want = np.fft.ifft(x) * n if d > 0 else np.fft.fft(x)
        assert np.abs(y - want).max() < 1e-12 * np.abs(want).max()


def test_eigensolver_against_scipy(oracle):
    import scipy.linalg

    lib = oracle.library()
    rng = np.random.default_rng(3)
    n = 40
    a = rng.normal(size=(n, n))
    a = a + a.T
    e = np.zeros(n)
    u = np.zeros((n, n))
    af = np.asfortranarray(a)
    uf = np.asfortranarray(u)
    lib.orc_syev(n, af.ctypes.data_as(C.POINTER(C.c_double)), e.ctypes.data_as(C.POINTER(C.c_double)),
                 uf.ctypes.data_as(C.POINTER(C.c_double)))
    assert np.abs(np.sort(e) - scipy.linalg.eigvalsh(a)).max() < 1e-12
    assert np.abs(a @ uf - uf * e[None, :]).max() < 1e-11


def test_initializerandom_deterministic(oracle):
    """WAVES_INITIALIZERANDOM: deterministic stream, envelope exp(-G^2/6)."""
    lib = oracle.library()
    s = systems.named_system("Si8")
    inp = systems.build_inputs(s)
    g = np.ascontiguousarray(inp["gvec"])
    out1 = np.zeros((4, inp["ngl"]), dtype=np.complex128)
    out2 = np.zeros_like(out1)
    dp = C.POINTER(C.c_double)
    lib.orc_initializerandom(inp["ngl"], 1, 4, g.ctypes.data_as(dp), out1.ctypes.data_as(dp))
    lib.orc_initializerandom(inp["ngl"], 1, 4, g.ctypes.data_as(dp), out2.ctypes.data_as(dp))
    assert np.array_equal(out1, out2)
    assert np.abs(out1).max() > 0
    env = np.exp(-0.5 * inp["g2"] / 3.0)
    assert np.all(np.abs(out1) <= 2 * env[None, :] + 1e-300)


def _band_overlap(inp, psi, proj):
    """Full NB x NB O-overlap of the real bands unravelled from super wave functions."""
    mg = inp["minusg"] - 1
    p1 = 0.5 * (psi + np.conj(psi[:, mg]))
    p2 = -0.5j * (psi - np.conj(psi[:, mg]))
    bands = np.empty((2 * len(psi), inp["ngl"]), complex)
    bands[0::2], bands[1::2] = p1, p2
    s = inp["omega"] * (np.conj(bands) @ bands.T)
    pr = np.empty((2 * len(psi), proj.shape[0]))
    pr[0::2], pr[1::2] = proj.real.T, proj.imag.T
    npro = proj.shape[0]
    D = np.zeros((npro, npro))
    ip = 0
    for a in range(inp["nat"]):
        sp = inp["isp"][a] - 1
        lox = inp["lox"][sp]
        dm = inp["dover"][sp].T
        offs, o = [], 0
        for l in lox:
            offs.append(o)
            o += 2 * l + 1
        for i, l1 in enumerate(lox):
            for j, l2 in enumerate(lox):
                if l1 == l2:
                    for m in range(2 * l1 + 1):
                        D[ip + offs[i] + m, ip + offs[j] + m] = dm[i, j]
        ip += o
    return (s + pr @ D @ pr.T).real


def test_oracle_orthonormality_and_drift(oracle):
    s = systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry")
    inp = systems.build_inputs(s)
    w = oracle.open_oracle(inp).setup().initialize()
    ov = _band_overlap(inp, w.download_psi(0), w.get_proj())
    # ORTHO_Y_C regularises its divisions by R8SMALL=1e-10 (src/paw_waves2.f90:1058)
    assert np.abs(ov - np.eye(inp["nb"])).max() < 1e-9
    w.set_dynamics(10.0, 0.3)
    for _ in range(20):
        w.cp_step()
    w.set_dynamics(10.0, 0.0)
    w.stop()
    psi0 = w.download_psi(0)
    proj0 = w.get_proj()
    drifts = []
    for dt in (10.0, 5.0):
        w.upload_psi(0, psi0)
        w.upload_psi(1, psi0)
        w.set_proj(proj0)
        w.set_rlam0(np.zeros((inp["nb"], inp["nb"]), complex))
        w.stop()
        w.set_dynamics(dt, 0.0)
        es = []
        for _ in range(int(60 / dt)):
            out, _ = w.cp_step()
            es.append(out[0] + out[2])
        drifts.append(np.ptp(es))
        ov = _band_overlap(inp, w.download_psi(0), w.get_proj())
        assert np.abs(ov - np.eye(inp["nb"])).max() < 1e-7  # ORTHO_X EPS 1e-8 on max|O-1|
    assert drifts[1] < drifts[0] / 2.5  # dt^2 scaling of the Verlet error


def test_golden_regression(oracle):
    """The oracle reproduces its committed fixtures (generated by tests/golden/make_golden.py)."""
    with open(os.path.join(GOLD, "oracle_si8_20ry.json")) as f:
        gold = json.load(f)
    from golden.make_golden import run_case  # noqa: E402

    got = run_case(oracle)
    assert got["ngl"] == gold["ngl"]
    assert got["igvec_sha256"] == gold["igvec_sha256"]
    # the fixtures hold for both summation orders of the oracle (ZGEMM of the
    # bundled OpenBLAS or the plain loops): after six CP steps they part by
    # about 1e-9 Ha of 76 Ha, so the bound is the energy tolerance of the path
    for k in ("etot", "ekin", "ekinpsi", "iters"):
        assert np.allclose(got[k], gold[k], rtol=0, atol=1e-8), k
    assert np.allclose(got["force0"], gold["force0"], rtol=0, atol=1e-8)


def _numpy_density(inp, psi, occ):
    """WAVES_DENSITY at Gamma by numpy: psi(r) = sum_G psi(G) exp(iGr) on the
    grid (x fastest), rho = sum f1 Re(psi)^2 + f2 Im(psi)^2."""
    nr1, nr2, nr3 = inp["grid"]
    ig = inp["igvec"]
    rho = np.zeros((nr3, nr2, nr1))
    for b in range(psi.shape[0]):
        grid = np.zeros((nr3, nr2, nr1), complex)
        grid[ig[:, 2] % nr3, ig[:, 1] % nr2, ig[:, 0] % nr1] = psi[b]
        r = np.fft.ifftn(grid) * grid.size
        f1 = occ[2 * b]
        f2 = occ[2 * b + 1] if 2 * b + 1 < len(occ) else 0.0
        rho += f1 * r.real ** 2 + f2 * r.imag ** 2
    return rho


def test_oracle_density_and_denmat(oracle):
    """WAVES_DENSITY against numpy's FFT; WAVES_DENMAT against a numpy
    restatement of its TINV sums; both matrices real and symmetric."""
    s = systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry")
    inp = systems.build_inputs(s)
    w = oracle.open_oracle(inp).setup().initialize()
    for _ in range(2):
        w.cp_step()
    rho = w.density()
    want = _numpy_density(inp, w.download_psi(0), inp["occ"])
    assert np.abs(rho - want).max() < 1e-12 * np.abs(want).max()
    d, e = w.denmat()
    proj = w.get_proj().T  # (nbh, npro) complex
    occ = inp["occ"]
    s1 = 0.5 * (occ[0::2] + occ[1::2])
    s2 = 0.5 * (occ[0::2] - occ[1::2])
    p0 = 0
    for a, isp in enumerate(inp["isp"].tolist()):
        lmnx = sum(2 * l + 1 for l in inp["lox"][isp - 1])
        p = proj[:, p0:p0 + lmnx]
        dm = np.einsum("bi,bj->ij", p, s1[:, None] * p.conj() + s2[:, None] * p).real
        dm = 0.5 * (dm + dm.T)
        assert np.abs(d[a][:lmnx, :lmnx].T - dm).max() < 1e-12 * max(1.0, np.abs(dm).max())
        assert np.abs(d[a].imag).max() == 0.0 and np.abs(e[a].imag).max() == 0.0
        assert np.abs(e[a] - e[a].T).max() < 1e-13 * max(1.0, np.abs(e[a]).max())
        p0 += lmnx


def test_oracle_restart_records(oracle, tmp_path):
    """WAVES$WRITE record layout, read back into a fresh set: the next steps
    are bit-identical; a file with its G vectors permuted and a part of them
    missing maps by G vector and zero-fills the rest (WAVES_READPSI)."""
    import restart_file as rf

    s = systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry")
    inp = systems.build_inputs(s)
    w = oracle.open_oracle(inp).setup().initialize()
    for _ in range(3):
        w.cp_step()
    p = tmp_path / "a.rst"
    w.write_restart(p, inp["rbas"])
    d = rf.parse_waves(rf.read_records(p))
    assert (d["id"], d["name"], d["version"], d["notes"]) == ("WAVES", "NONE", "AUG1996", "NONE")
    assert (d["nkpt"], d["nspin"], d["nwave"], d["ndim"], d["tsuper"]) == (1, 1, 2, 1, 1)
    assert d["ngg"] == w.ngl and d["nb"] == w.nb and d["nlambda"] == 2
    assert np.array_equal(d["rbas"], np.asarray(inp["rbas"], dtype=np.float64))
    assert np.array_equal(d["igvec"], np.asarray(inp["igvec"]).reshape(-1, 3))
    assert np.array_equal(d["psi"][0], w.download_psi(0))
    assert np.array_equal(d["psi"][1], w.download_psi(1))
    assert np.array_equal(d["lambda"][0], w.get_rlam0())
    # RBAS from the handle's GBAS when none is given
    q = tmp_path / "b.rst"
    w.write_restart(q)
    r2 = rf.parse_waves(rf.read_records(q))["rbas"]
    assert np.abs(r2 - np.asarray(inp["rbas"])).max() < 1e-12 * np.abs(inp["rbas"]).max()

    v = oracle.open_oracle(inp).setup()
    v.read_restart(p)
    assert np.array_equal(v.download_psi(0), w.download_psi(0))
    assert np.array_equal(v.download_psi(1), w.download_psi(1))
    # PROJ is not in the file: both form it from PSI0, as a run does at its
    # first step (WAVES$ETOT at TFIRST)
    w.projections()
    v.projections()
    for _ in range(2):
        ea, eb = w.cp_step(), v.cp_step()
    assert np.array_equal(w.download_psi(0), v.download_psi(0))
    assert np.array_equal(ea[0], eb[0]) and np.array_equal(ea[1], eb[1])

    # permuted and truncated G set
    rng = np.random.default_rng(7)
    perm = rng.permutation(d["ngg"])
    keep = d["ngg"] - 50
    rf.write_records(tmp_path / "c.rst", rf.permuted(rf.read_records(p), perm, keep))
    u = oracle.open_oracle(inp).setup()
    u.read_restart(tmp_path / "c.rst")
    want0, want1 = d["psi"][0].copy(), d["psi"][1].copy()
    want0[:, perm[keep:]] = 0.0
    want1[:, perm[keep:]] = 0.0
    assert np.array_equal(u.download_psi(0), want0)
    assert np.array_equal(u.download_psi(1), want1)
    # a static restart (NWAVE = 1) starts PSIM from PSI0
    rf.write_records(tmp_path / "s.rst", rf.static(rf.read_records(p)))
    t = oracle.open_oracle(inp).setup()
    t.read_restart(tmp_path / "s.rst")
    assert np.array_equal(t.download_psi(0), d["psi"][0])
    assert np.array_equal(t.download_psi(1), d["psi"][0])
    # a file cut inside a wave-function record is refused
    raw = p.read_bytes()
    (tmp_path / "cut.rst").write_bytes(raw[: len(raw) // 2])
    u2 = oracle.open_oracle(inp).setup()
    u2.read_restart(p)
    with pytest.raises(Exception):
        u2.read_restart(tmp_path / "cut.rst")
    assert np.array_equal(u2.download_psi(0), d["psi"][0])  # left as it was
    # a file of another band count is refused
    bad = rf.read_records(p)
    import struct
    bad[2] = bad[2][:16] + struct.pack("<i", w.nb + 2) + bad[2][20:]
    rf.write_records(tmp_path / "d.rst", bad)
    with pytest.raises(Exception):
        oracle.open_oracle(inp).setup().read_restart(tmp_path / "d.rst")
    # a negative G-vector count and a record marker of 2 GB are refused as
    # argument errors, before anything is sized from them
    for name, raw in rf.damaged(p):
        (tmp_path / name).write_bytes(raw)
        with pytest.raises(Exception):
            u2.read_restart(tmp_path / name)
        assert np.array_equal(u2.download_psi(0), d["psi"][0])



# ---------------------------------------------------------------------------
# POTENTIAL$VOFRHO.  The reference checks this routine with its own self-tests
# (POTENTIAL_VOFRHO, src/paw_potential.f90:619-650 and 860-880, SELFTEST
# ITEST = 1, 2, 3): the potential is the derivative of EHARTREE + EXC with
# respect to the density, VQLM the derivative with respect to QLM, the forces
# minus the derivative with respect to the positions.  The same three checks
# by central differences pin the oracle's restatement; a numpy restatement of
# the formulas checks its arithmetic.
# ---------------------------------------------------------------------------
def _vofrho_case(oracle):
    inp = systems.build_inputs(systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=15.0, name="Si8-15", disp=0.1))
    w = oracle.open_oracle(inp).setup().initialize()
    w.set_rhoset()
    return inp, w


def test_oracle_vofrho_selftests(oracle):
    inp, w = _vofrho_case(oracle)
    rho = w.density()
    v, e, f, vq = w.vofrho(rho)
    om, nr = inp["omega"], rho.size

    def energy(r=rho, q=None):
        _, ee, _, _ = w.vofrho(r, q)
        return ee["ehartree"] + ee["exc"]

    # ITEST 1: dE/drho along a seeded in-sphere direction equals int V drho
    n = tuple(inp["grid"])
    ig = inp["rhoset"]["igvec"]
    mask = np.zeros(n, bool)
    for sgn in (1, -1):
        mask[(sgn * ig[:, 0]) % n[0], (sgn * ig[:, 1]) % n[1], (sgn * ig[:, 2]) % n[2]] = True
    rng = np.random.default_rng(1)
    spec = rng.normal(size=n) + 1j * rng.normal(size=n)
    dr = np.fft.ifftn(np.where(mask, spec, 0)).real.transpose(2, 1, 0) * 100
    d = 1e-4
    fd = (energy(rho + d * dr) - energy(rho - d * dr)) / (2 * d)
    assert abs(fd - (v * dr).sum() * om / nr) < 1e-6 * max(1.0, abs(fd))
    # a single grid point
    k = (5, 7, 3)
    rp, rm = rho.copy(), rho.copy()
    rp[k] += 1e-5
    rm[k] -= 1e-5
    assert abs((energy(rp) - energy(rm)) / 2e-5 / (om / nr) - v[k]) < 1e-6 * abs(v[k])
    # ITEST 2: VQLM = dE/dQLM
    q0 = inp["rhoset"]["qlm"].copy()
    for a, lm in ((0, 0), (3, 2), (5, 7)):
        qp, qm = q0.copy(), q0.copy()
        qp[a, lm] += 1e-5
        qm[a, lm] -= 1e-5
        fdq = (energy(rho, qp) - energy(rho, qm)) / 2e-5
        assert abs(fdq - vq[a, lm]) < 1e-6 * max(1e-2, abs(vq[a, lm])), (a, lm, fdq, vq[a, lm])
    w.set_qlm(q0)
    # ITEST 3: forces = -dE/dR
    r0 = inp["r0"].copy()
    for a, c in ((0, 0), (3, 2), (6, 1)):
        rp = r0.copy()
        rp[a, c] += 1e-5
        w.set_atoms(rp, None)
        ep = energy()
        rm = r0.copy()
        rm[a, c] -= 1e-5
        w.set_atoms(rm, None)
        em = energy()
        assert abs(-(ep - em) / 2e-5 - f[a, c]) < 1e-6 * max(1.0, abs(f[a, c])), (a, c)
    w.set_atoms(r0, None)


def test_oracle_vofrho_matches_numpy(oracle):
    """The potential formulas restated once more in numpy (full-grid FFTs,
    direct structure factors)."""
    inp, w = _vofrho_case(oracle)
    rho = w.density()
    v, e, _, _ = w.vofrho(rho)
    R = inp["rhoset"]
    n = tuple(inp["grid"])
    om, N = inp["omega"], rho.size
    ig, g, g2, y, q = R["igvec"], R["gvec"], R["g2"], R["ylm"], R["qlm"]
    y0 = 1 / np.sqrt(4 * np.pi)
    ip = tuple((ig[:, k] % n[k]) for k in range(3))
    im = tuple((-ig[:, k] % n[k]) for k in range(3))

    def rtog(f):
        F = np.fft.fftn(f.transpose(2, 1, 0)) / N
        return 0.5 * (F[ip] + np.conj(F[im]))

    def gtor(c):
        F = np.zeros(n, complex)
        F[ip] = c
        F[im] = np.conj(c)
        return (np.fft.ifftn(F) * N).real.transpose(2, 1, 0)

    cfac = np.array([1] + [-1j / 3] * 3 + [-1 / 15] * 5)
    ng = int(np.nonzero((ig == 0).all(1))[0][0])
    isp = inp["isp"] - 1
    eig = [np.exp(-1j * (g @ r)) for r in inp["r0"]]
    rhog = rtog(rho)
    for a in range(len(eig)):
        rhog = rhog + R["pscore"][isp[a]] * y0 * eig[a]
    rho2, pot, vb = rhog.copy(), np.zeros_like(rhog), 0.0
    for a in range(len(eig)):
        s = isp[a]
        c = (y * (cfac * q[a])[None, :]).sum(1) * eig[a]
        vb += q[a, 0] * y0 * R["v0"][s][ng]
        rho2 = rho2 + c * R["g0"][s]
        pot = pot + c * R["v0"][s] + R["vbar"][s] * y0 * eig[a]
    rhob = -rho2[ng].real
    rho2[ng] = 0
    gs = np.where(np.arange(len(g2)) == ng, 1, g2)
    vg = rho2 * 4 * np.pi / gs
    vg[ng] = -vb
    terms = 0.5 * np.conj(rho2) * vg + np.conj(rhog) * pot
    terms[ng] = 0.5 * (np.conj(rhog[ng]) * pot[ng] + rhob * vb)
    eh = terms.sum().real * 2 * om
    rt = np.maximum(gtor(rhog), 1e-8)
    ex = -3 / (4 * np.pi) * (3 * np.pi ** 2) ** (1 / 3) * rt ** (4 / 3)
    au, a1, b1, b2, b3, b4 = 3.10907e-2, 2.1370e-1, 7.5957, 3.5876, 1.6382, 4.9294e-1
    rs = (3 / (4 * np.pi)) ** (1 / 3) / rt ** (1 / 3)
    sq = np.sqrt(rs)
    s1, ds1 = -2 * au * (1 + a1 * rs), -2 * au * a1
    s2 = 2 * au * sq * (b1 + b2 * sq + b3 * rs + b4 * rs * sq)
    ds2 = au / sq * (b1 + 2 * b2 * sq + 3 * b3 * rs + 4 * b4 * rs * sq)
    s3 = 1 + 1 / s2
    ecu = s1 * np.log(s3)
    decu = (ds1 * np.log(s3) + s1 * (-ds2 / s2 ** 2) / s3) * (-rs / 3 / rt)
    exc = (ex + rt * ecu).sum() * om / N
    vxc = ex * 4 / 3 / rt + rt * decu + ecu
    vnp = gtor(rtog(vxc) + pot + vg)
    assert abs(eh - e["ehartree"]) < 1e-10 * abs(eh)
    assert abs(exc - e["exc"]) < 1e-10 * abs(exc)
    assert abs(rhob - e["rhob"]) < 1e-12
    assert np.abs(vnp - v).max() < 1e-10 * np.abs(v).max()


def _ortho_y_c(oracle, phiphi, chiphi, chichi, smap=None):
    """orc_ortho_y_c: WAVES_ORTHO_Y_C of the oracle on complex NB x NB matrices."""
    lib = oracle.library()
    f = lib.orc_ortho_y_c
    f.restype = C.c_int
    f.argtypes = [C.c_int] + [C.c_void_p] * 5
    nb = phiphi.shape[0]
    mats = [np.asfortranarray(m, dtype=np.complex128) for m in (phiphi, chiphi, chichi)]
    x = np.zeros((nb, nb), dtype=np.complex128, order="F")
    mp = None if smap is None else np.ascontiguousarray(smap, dtype=np.int32)
    rc = f(nb, *[m.ctypes.data for m in mats], x.ctypes.data, None if mp is None else mp.ctypes.data)
    return rc, x


@pytest.mark.parametrize("order", ["identity", "permuted"])
@pytest.mark.parametrize("kind", ["complex", "real"])
def test_oracle_ortho_y_c_self_test(oracle, order, kind):
    """WAVES_ORTHO_Y_C (src/paw_waves2.f90:1025-1338) against the reference's
    own TTEST checks of the routine (:1302-1336, TESTA :1343-1356): with
    |phi'_I> = |phi_I> + sum_J |chi_J> X(J,I), PHIPHI + X^H CHIPHI + CHIPHI^H X
    + X^H CHICHI X = 1 (the reference stops above TOL = 1e-10; its divisions
    carry R8SMALL = 1e-10, :1058), and X(I,J) = 0 where I comes after J in
    the order MAP (the states are orthonormalised one after another)."""
    rng = np.random.default_rng(11)
    nb, ng = 12, 300
    cz = 1j if kind == "complex" else 0.0
    q, _ = np.linalg.qr(rng.normal(size=(ng, nb)) + cz * rng.normal(size=(ng, nb)))
    # columns of norm about 1 with perturbations of norm about 0.1 and 0.05
    phi = q + 0.1 / np.sqrt(ng) * (rng.normal(size=(ng, nb)) + cz * rng.normal(size=(ng, nb)))
    chi = q + 0.05 / np.sqrt(ng) * (rng.normal(size=(ng, nb)) + cz * rng.normal(size=(ng, nb)))
    phiphi = phi.conj().T @ phi
    chiphi = chi.conj().T @ phi  # CHIPHI(I,J) = <chi_I|phi_J>
    chichi = chi.conj().T @ chi
    smap = np.arange(nb) if order == "identity" else rng.permutation(nb)
    rc, x = _ortho_y_c(oracle, phiphi, chiphi, chichi, None if order == "identity" else smap)
    assert rc == 0
    res = phiphi + x.conj().T @ chiphi + chiphi.conj().T @ x + x.conj().T @ chichi @ x - np.eye(nb)
    assert np.abs(res).max() < 1e-9
    new = phi + chi @ x
    assert np.abs(new.conj().T @ new - np.eye(nb)).max() < 1e-9
    pos = np.empty(nb, int)
    pos[smap] = np.arange(nb)
    later = pos[:, None] > pos[None, :]
    assert np.all(x[later] == 0) and np.abs(x[~later]).max() > 0
    if kind == "real":
        assert np.all(x.imag == 0)


def test_oracle_safeortho_false(oracle):
    """WAVES$ORTHOGONALIZE with SAFEORTHO = F (src/paw_waves2.f90:306-386):
    WAVES_ORTHO_Y_C of MAT, OMAT, OOMAT replaces WAVES_ORTHO_X, with SMAP
    sorting the states by the RLAM0 diagonal when SWAPSTATES = T.  The CP
    steps keep PSI orthonormal (O-metric) and report no iterations; the state
    order changes the result."""
    s = systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry")
    inp = systems.build_inputs(s)
    w = oracle.open_oracle(inp).setup().initialize()
    for _ in range(3):
        w.cp_step()
    state = (w.download_psi(0), w.download_psi(1), w.get_proj(), w.get_rlam0())
    d = np.diag(state[3]).real
    assert not np.all(np.diff(d) >= 0)  # the sort has something to do
    results = {}
    for swap in (0, 1):
        w.upload_psi(0, state[0])
        w.upload_psi(1, state[1])
        w.set_proj(state[2])
        w.set_rlam0(state[3])
        w.set_option(8, swap)  # CUW_OPT_SWAPSTATES
        w.set_option(7, 0)  # CUW_OPT_SAFEORTHO = F
        for _ in range(3):
            out, _ = w.cp_step()
            assert out[4] == 0
            ov = _band_overlap(inp, w.download_psi(0), w.get_proj())
            # R8SMALL = 1e-10 in the divisions of ORTHO_Y_C (waves2:1058), here
            # against CHICHI = <O psi|O psi> (dt^2/m)^2 of order 1e-2
            assert np.abs(ov - np.eye(inp["nb"])).max() < 1e-8
        results[swap] = w.download_psi(0)
    assert np.abs(results[0] - results[1]).max() > 1e-6
    w.set_option(7, 1)
    out, _ = w.cp_step()
    assert out[4] > 0


def test_oracle_cell_friction_propagate(oracle):
    """WAVES$PROPAGATE with TSTRESS (src/paw_waves1.f90:6524-6543): the oracle's
    per-G coefficients from WAVES_DMPSI (:6676-6711) against a numpy
    restatement of the two routines (the reference reads the upper triangle of
    FRICMAT, so a non-symmetric matrix checks the index order); switching the
    friction off gives back the scalar path bit for bit."""
    s = systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry")
    inp = systems.build_inputs(s)
    w = oracle.open_oracle(inp).setup().initialize()
    rng = np.random.default_rng(4)
    f = rng.normal(size=(3, 3)) * 2e-5  # a strain rate times DELT/2
    db = rng.uniform(0.0, 0.2, size=inp["ngl"])
    annee = 0.05
    w.set_dynamics(inp["delt"], annee)
    psi0, psim = w.download_psi(0), w.download_psi(1)
    w.hpsi()
    hp = w.download_psi(2)
    x, y, z = inp["gvec"].T
    svar = (f[0, 0] * x * x + 2 * f[0, 1] * x * y + 2 * f[0, 2] * x * z + f[1, 1] * y * y
            + 2 * f[1, 2] * y * z + f[2, 2] * z * z)
    an = annee - 0.5 * np.trace(f) - inp["emass"] * inp["emasscg2"] * svar * (1.0 + db)
    want = (2.0 / (1.0 + an)) * psi0 + (1.0 - 2.0 / (1.0 + an)) * psim \
        - inp["delt"] ** 2 / (1.0 + an) / inp["mpsi"] * hp
    w.set_cell_friction(f, inp["emass"], inp["emasscg2"], db)
    w.propagate()
    got = w.download_psi(1)
    assert np.abs(got - want).max() / np.abs(want).max() < 1e-13
    # off again: the scalar ANNEE path
    w.upload_psi(1, psim)
    w.set_cell_friction(None)
    w.hpsi()
    w.propagate()
    a1 = 2.0 / (1.0 + annee)
    plain = a1 * psi0 + (1.0 - a1) * psim - inp["delt"] ** 2 / (1.0 + annee) / inp["mpsi"] * hp
    assert np.abs(w.download_psi(1) - plain).max() / np.abs(plain).max() < 1e-13
