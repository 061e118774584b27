"""The serving runtime (cuwaves_server_*) on the GPU.

A request's result (energies, forces after its last step) must be bit for bit
the same whether it runs alone or mixed with other requests of other sizes,
precisions and step counts, and the same as the single-system path of the
engine; the single point (cuwaves_etot) matches the oracle within the FP64
tolerances of the parity tests (1e-8 Ha, 1e-6 Ha/bohr).  Admission keeps the
admitted device memory within the budget.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import cuwaves  # noqa: E402
from cuwaves import CUW_PREC_FP64, CUW_PREC_MIXED, CUW_PSI0, CUW_PSIM, systems  # noqa: E402
from cuwaves.serve import Server  # noqa: E402

CASES = {
    "Si2mol": lambda: systems.molecule_box("Si2", box=12.0, epw_psi_ry=15.0, grid=(20, 20, 20)),
    "Si6": lambda: systems.si_small(6, epw_psi_ry=15.0, grid=(20, 20, 20)),
    "H2O2": lambda: systems.water_box(2, box=10.0, lattice=(2, 1, 1), epw_psi_ry=25.0, grid=(32, 32, 32)),
    "Si8-20Ry": lambda: systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry"),
}

# (system, nsteps, move atoms, precision); nsteps 0 is a single point
MIX = [
    ("Si2mol", 0, False, CUW_PREC_FP64),
    ("Si6", 3, True, CUW_PREC_FP64),
    ("H2O2", 0, False, CUW_PREC_FP64),
    ("Si8-20Ry", 4, False, CUW_PREC_FP64),
    ("Si8-20Ry", 3, True, CUW_PREC_MIXED),
    ("H2O2", 2, True, CUW_PREC_MIXED),
    ("Si6", 0, False, CUW_PREC_FP64),
]


@pytest.fixture(scope="module")
def inputs():
    return {name: systems.build_inputs(make()) for name, make in CASES.items()}


def run_alone(inp, nsteps, move, prec):
    srv = Server(hbm_budget=16 << 30, workers=1)
    try:
        rid = srv.submit(inp, nsteps=nsteps, move_atoms=move, precision=prec)
        _, out, f, _ = srv.result(rid)
        return out, f, srv.stats()
    finally:
        srv.close()


def test_result_alone_equals_result_in_the_mix(inputs):
    alone = [run_alone(inputs[s], n, m, p)[:2] for s, n, m, p in MIX]
    srv = Server(hbm_budget=16 << 30, workers=4)
    try:
        ids = [srv.submit(inputs[s], nsteps=n, move_atoms=m, precision=p) for _ in range(2) for s, n, m, p in MIX]
        assert srv.wait_all() == 0
        for k, rid in enumerate(ids):
            st, out, f, lat = srv.poll(rid)
            ref_out, ref_f = alone[k % len(MIX)]
            assert st == 0
            assert lat > 0.0
            assert np.array_equal(out, ref_out), (MIX[k % len(MIX)], out, ref_out)
            assert np.array_equal(f, ref_f), MIX[k % len(MIX)]
        s = srv.stats()
        assert s["completed"] == len(ids) and s["failed"] == 0
        assert s["mean_admitted"] > 1.0  # the requests did overlap
        assert s["p99_ms"] >= s["p50_ms"] > 0.0
    finally:
        srv.close()


def test_server_matches_single_system_path_and_oracle(inputs, oracle):
    inp = inputs["Si6"]
    # single point: server vs engine vs oracle
    out_s, f_s, _ = run_alone(inp, 0, False, CUW_PREC_FP64)
    w = cuwaves.open_waves(inp).setup().initialize()
    e_d, f_d = w.etot()
    assert np.array_equal(out_s[:2], e_d) and np.array_equal(f_s, f_d)
    cpu = oracle.open_oracle(inp).setup()
    for which in (CUW_PSI0, CUW_PSIM):
        cpu.upload_psi(which, w.download_psi(which))
    cpu.set_proj(w.get_proj())
    e_c, f_c = cpu.etot()
    assert np.abs(e_d - e_c).max() < 1e-8, (e_d, e_c)
    assert np.abs(f_d - f_c).max() < 1e-6
    # CP steps with moving nuclei: server vs engine
    out_s, f_s, _ = run_alone(inp, 3, True, CUW_PREC_FP64)
    w = cuwaves.open_waves(inp).setup().initialize()
    for _ in range(3):
        out_d, f_d = w.cp_step(move_atoms=True)
    assert np.array_equal(out_s, out_d) and np.array_equal(f_s, f_d)


def test_admission_keeps_memory_within_budget(inputs):
    inp = inputs["Si8-20Ry"]
    one = run_alone(inp, 1, False, CUW_PREC_FP64)[2]["peak_bytes"]
    assert one > 0
    budget = int(2.5 * one)  # room for two sets at a time
    srv = Server(hbm_budget=budget, workers=4)
    try:
        ids = [srv.submit(inp, nsteps=2) for _ in range(6)]
        assert srv.wait_all() == 0
        s = srv.stats()
        assert s["completed"] == 6 and s["failed"] == 0
        assert one * 2 <= s["peak_bytes"] <= budget
        assert s["mean_admitted"] <= 2.0 + 1e-9
        outs = [srv.poll(r)[1] for r in ids]
        assert all(np.array_equal(o, outs[0]) for o in outs)
    finally:
        srv.close()


def test_estimate_bounds_the_allocation(inputs):
    """The admission estimate is at least the device memory a set really holds
    (handle, FFT work grid and contraction scratch after a CP step)."""
    import torch

    inp = inputs["H2O2"]
    est = run_alone(inp, 1, False, CUW_PREC_FP64)[2]["peak_bytes"]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    w = cuwaves.open_waves(inp).setup().initialize()
    w.cp_step()
    free1 = torch.cuda.mem_get_info()[0]
    w.close()
    assert free0 - free1 <= est, (free0 - free1, est)


def test_handles_of_different_grids_interleave():
    """Kernel launch limits are per function and shared by every handle: a set
    created after a larger one must not break the larger one's next step."""
    big = systems.build_inputs(systems.molecule_box("H2O", box=20.0))         # 56^3 grid
    small = systems.build_inputs(systems.si_small(2))                        # 28^3 grid
    tall = systems.build_inputs(systems.si_small(12))                        # 28 x 28 x 56
    for prec in (CUW_PREC_FP64, CUW_PREC_MIXED):
        a = cuwaves.open_waves(big, precision=prec).setup().initialize()
        a.cp_step(move_atoms=True)
        b = cuwaves.open_waves(small, precision=prec).setup().initialize()
        c = cuwaves.open_waves(tall, precision=prec).setup().initialize()
        for _ in range(2):
            for w in (a, b, c):
                w.cp_step(move_atoms=True)
        for w in (a, b, c):
            w.close()


def test_concurrent_sets_match_alone():
    """Mixed-precision sets of serving size stepped at the same time from
    several host threads (each on its own stream, so that the kernels of
    different sets share the SMs) give bit for bit the results of the same
    sets run one at a time."""
    import threading

    specs = [("Si", 32, 1), ("W", 8, 1), ("Si", 64, 1), ("W", 4, 2), ("Si", 16, 1), ("Si", 32, 2), ("W", 16, 1)]
    inps = [systems.build_inputs(systems.serving_system(k, n, s)) for k, n, s in specs]
    nsteps = 4

    def run(inp, out, i):
        w = cuwaves.open_waves(inp, precision=CUW_PREC_MIXED).setup().initialize()
        res = []
        for _ in range(nsteps):
            o, f = w.cp_step(move_atoms=True)
            res.append((o.copy(), f.copy()))
        w.close()
        out[i] = res

    alone = [None] * len(inps)
    for i, inp in enumerate(inps):
        run(inp, alone, i)
    for _ in range(2):
        mixed = [None] * len(inps)
        th = [threading.Thread(target=run, args=(inp, mixed, i)) for i, inp in enumerate(inps)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for i, spec in enumerate(specs):
            assert mixed[i] is not None, spec
            for step, ((oa, fa), (om, fm)) in enumerate(zip(alone[i], mixed[i])):
                assert np.array_equal(oa, om) and np.array_equal(fa, fm), (spec, step)


def test_stream_priority_keeps_results(inputs):
    """CUW_OPT_STREAM_PRIORITY replaces the handle's stream (after the work in
    flight) and retires its step graphs; the steps give bit for bit the same
    energies and forces on the high- and the low-priority stream."""
    inp = inputs["Si8-20Ry"]
    outs = []
    for prio in (0, 1):
        w = cuwaves.open_waves(inp, precision=CUW_PREC_MIXED).setup().initialize()
        w.cp_step(move_atoms=True)
        w.set_option(cuwaves.CUW_OPT_STREAM_PRIORITY, prio)
        res = [w.cp_step(move_atoms=True) for _ in range(3)]
        w.set_option(cuwaves.CUW_OPT_STREAM_PRIORITY, 1 - prio)
        res.append(w.cp_step(move_atoms=True))
        outs.append(res)
        w.close()
    for (o0, f0), (o1, f1) in zip(outs[0], outs[1]):
        assert np.array_equal(o0, o1) and np.array_equal(f0, f1)
    w = cuwaves.open_waves(inp).setup()
    with pytest.raises(cuwaves.WavesError):
        w.set_option(cuwaves.CUW_OPT_STREAM_PRIORITY, 2)
    w.close()
