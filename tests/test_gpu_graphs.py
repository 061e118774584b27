"""CP steps replayed as CUDA graphs (CUW_OPT_GRAPHS) against the same steps
launched kernel by kernel: bit-identical energies, forces and wave functions,
through the PSI0/PSIM buffer swap and the position updates, through a change
of the dynamics between steps (which retires the graphs), through per-step
position uploads (the e2e loop of the bench), and through the rediagonalisation
that follows a failed Lyapunov fixed point, which is decided on the device.
No reference counterpart: the reference has no device launches to record."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import cuwaves  # noqa: E402
from cuwaves import (CUW_OPT_GRAPHS, CUW_OPT_LYAP_MAX_SWEEPS, CUW_PREC_FP64, CUW_PREC_MIXED, CUW_PSI0,  # noqa: E402
                     systems)

CASES = {
    "Si8-20Ry": lambda: systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry"),
    "H2O2": lambda: systems.water_box(2, box=10.0, lattice=(2, 1, 1), epw_psi_ry=25.0, grid=(32, 32, 32)),
}


@pytest.fixture(scope="module")
def inputs():
    return {name: systems.build_inputs(make()) for name, make in CASES.items()}


def twins(inp, prec, opts=None):
    ws = []
    for graphs in (1, 0):
        w = cuwaves.open_waves(inp, precision=prec)
        w.set_option(CUW_OPT_GRAPHS, graphs)
        for k, v in (opts or {}).items():
            w.set_option(k, v)
        ws.append(w.setup().initialize())
    return ws


def same_step(ga, gb, move=True):
    oa, fa = ga.cp_step(move_atoms=move)
    ob, fb = gb.cp_step(move_atoms=move)
    assert np.array_equal(oa, ob), (oa, ob)
    assert np.array_equal(fa, fb)


@pytest.mark.parametrize("prec", [CUW_PREC_FP64, CUW_PREC_MIXED])
@pytest.mark.parametrize("name", sorted(CASES))
def test_graph_steps_equal_launched_steps(inputs, name, prec):
    ga, gb = twins(inputs[name], prec)
    for _ in range(9):
        same_step(ga, gb)
    n, replays = ga.graph_stats()
    assert 1 <= n <= 2 and replays >= 5
    assert gb.graph_stats() == (0, 0)
    # a change of the dynamics retires the graphs; positions uploaded every
    # step (EIGR rebuilt) take graphs of their own
    for w in (ga, gb):
        w.set_dynamics(8.0, 0.02)
    for _ in range(8):
        for w in (ga, gb):
            w.set_atoms(w.get_atoms()[1])
        same_step(ga, gb)
    assert ga.graph_stats()[1] > replays
    assert np.array_equal(ga.download_psi(CUW_PSI0), gb.download_psi(CUW_PSI0))
    ga.close()
    gb.close()


def test_rediagonalisation_inside_graphs(inputs):
    """One sweep per Lyapunov solve: the fixed point fails in every step and
    the gated rediagonalisation runs inside the replayed graphs."""
    ga, gb = twins(inputs["Si8-20Ry"], CUW_PREC_FP64, {CUW_OPT_LYAP_MAX_SWEEPS: 1})
    for _ in range(8):
        same_step(ga, gb)
    assert ga.graph_stats()[1] >= 2
    sa, sb = ga.ortho_stats(), gb.ortho_stats()
    assert sa["fixed_point_fallbacks"] >= 6 and sa == sb
    ga.close()
    gb.close()


@pytest.mark.parametrize("prec", [CUW_PREC_FP64, CUW_PREC_MIXED])
def test_async_input_copies_follow_enqueued_work(inputs, prec):
    """In asynchronous mode a new potential is copied in stream order: H|psi>
    calls enqueued before cuwaves_set_potential still see the old V(r), and
    the next one sees the new V(r); in both cases bit for bit what synchronous
    calls give."""
    inp = inputs["Si8-20Ry"]
    w = cuwaves.open_waves(inp, precision=prec).setup().initialize()
    v1 = np.ascontiguousarray(inp["v"], dtype=np.float64)
    v2 = v1 * 1.25 + 0.05
    w.set_potential(v2)
    w.projections()
    w.hpsi()
    want2 = w.expectation()
    w.set_potential(v1)
    w.hpsi()
    want1 = w.expectation()
    assert not np.array_equal(want1, want2)
    w.set_async(True)
    for _ in range(6):  # several milliseconds of queued work ahead of the copy
        w.hpsi()
    w.set_potential(v2)
    w.set_async(False)
    w.synchronize()
    assert np.array_equal(w.expectation(), want1)
    w.hpsi()
    assert np.array_equal(w.expectation(), want2)
    w.close()
