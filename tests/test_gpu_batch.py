"""Sets of uneven size advanced together by one CUDA graph launch
(cuwaves_batch_step) give bit for bit the results of stepping each set alone
with cuwaves_cp_step: the batch graph holds each set's own launches in their
own order, on its own stream."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import cuwaves  # noqa: E402
from cuwaves import CUW_PREC_FP64, CUW_PREC_MIXED, CUW_PSI0, CUW_PSIM, systems  # noqa: E402

MIX = [
    lambda: systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry"),
    lambda: systems.water_box(2, box=10.0, lattice=(2, 1, 1), epw_psi_ry=25.0, grid=(32, 32, 32)),
    lambda: systems.si_small(6, epw_psi_ry=15.0, grid=(20, 20, 20)),
    lambda: systems.molecule_box("Si2", box=12.0, epw_psi_ry=15.0, grid=(20, 20, 20)),
]


def pairs(precision, share=0):
    out = []
    for make in MIX:
        inp = systems.build_inputs(make())
        a = cuwaves.open_waves(inp, precision=precision).setup().initialize()
        b = cuwaves.open_waves(inp, precision=precision).setup()
        for w in (a, b):
            w.set_option(cuwaves.CUW_OPT_SM_SHARE, share)
        for which in (CUW_PSI0, CUW_PSIM):
            b.upload_psi(which, a.download_psi(which))
        b.set_proj(a.get_proj())
        b.set_rlam0(a.get_rlam0())
        for w in (a, b):
            w.cp_step(move_atoms=True)  # the eigenbasis and the Lagrange history
        out.append((inp, a, b))
    return out


@pytest.mark.parametrize("precision,share", [(CUW_PREC_FP64, 0), (CUW_PREC_MIXED, 0), (CUW_PREC_FP64, 4),
                                             (CUW_PREC_MIXED, 4)])
def test_batch_equals_sets_alone(precision, share):
    """share: CUW_OPT_SM_SHARE of every set (0: the whole device), the same for
    the set in the batch and its twin stepped alone."""
    ps = pairs(precision, share)
    batch = cuwaves.Batch([a for _, a, _ in ps])
    for rep in range(3):  # the first call captures, the others replay
        out = batch.step(move_atoms=True)
        for i, (inp, a, b) in enumerate(ps):
            for s in range(2):
                ob, _ = b.cp_step(move_atoms=True)
                assert np.array_equal(out[i, s], ob), (rep, i, s, out[i, s], ob)
    for inp, a, b in ps:
        assert np.array_equal(a.download_psi(CUW_PSI0), b.download_psi(CUW_PSI0))
        assert np.array_equal(a.get_rlam0(), b.get_rlam0())
        ra, rb = a.get_atoms(), b.get_atoms()
        assert all(np.array_equal(x, y) for x, y in zip(ra, rb))
    # the sets remain usable one by one after the batch
    for inp, a, b in ps:
        oa, _ = a.cp_step(move_atoms=True)
        ob, _ = b.cp_step(move_atoms=True)
        assert np.array_equal(oa, ob)
    batch.close()


def test_batch_refuses_fresh_set():
    inp = systems.build_inputs(MIX[0]())
    w = cuwaves.open_waves(inp).setup().initialize()
    batch = cuwaves.Batch([w])
    with pytest.raises(cuwaves.WavesError) as e:
        batch.step()
    assert e.value.code == 3
    batch.close()


@pytest.mark.parametrize("precision,tol", [(CUW_PREC_FP64, 1e-11), (CUW_PREC_MIXED, 1e-6)])
def test_sm_share_changes_rounding_only(precision, tol):
    """A set whose launch shapes assume 4 SMs (CUW_OPT_SM_SHARE) takes other
    split-K factors and persistent grids than one that assumes the whole
    device: the same CP steps to rounding level (relative to the energy)."""
    inp = systems.build_inputs(MIX[0]())
    a = cuwaves.open_waves(inp, precision=precision).setup().initialize()
    b = cuwaves.open_waves(inp, precision=precision).setup()
    for which in (CUW_PSI0, CUW_PSIM):
        b.upload_psi(which, a.download_psi(which))
    b.set_proj(a.get_proj())
    b.set_option(cuwaves.CUW_OPT_SM_SHARE, 4)
    for _ in range(3):
        (oa, fa), (ob, fb) = a.cp_step(move_atoms=True), b.cp_step(move_atoms=True)
        assert oa[4] == ob[4]
        assert abs(oa[0] - ob[0]) <= tol * abs(oa[0])
        assert np.abs(fa - fb).max() < 1e-6
    with pytest.raises(cuwaves.WavesError):
        b.set_option(cuwaves.CUW_OPT_SM_SHARE, -1)
    a.close()
    b.close()
