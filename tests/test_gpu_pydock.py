"""pyDock-style elec + LJ energy and its adjoint on the GPU, against the FP64 oracle and central
finite differences (project-defined scoring; no reference counterpart).

Bars: FP64 energies within 1e-10 relative (summation order differs), FP32 within 1e-5;
FP32 and FP64 gradients within 1e-4 of the FP64 oracle gradient (max-norm relative);
FP64 gradient against central differences (h = 1e-4) within 1e-4 (the differences carry O(h^2) error)."""
import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import OracleState, OracleSystem, oracle_scores, oracle_step
from pydock_util import fd_grad, oracle_energy, oracle_grad

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cx():
    return sd.SyntheticComplex(757, 481, 2, 24, seed=41)


def test_pydock_energies(cx, tables):
    osys = OracleSystem(cx, tables, scoring=1)
    poses = cx.poses.reshape(-1, cx.pose_len)
    ref = np.array([oracle_energy(osys, p) for p in poses])
    with sd.Docking([cx], tables, scoring=sd.SD_SCORING_PYDOCK) as dk:
        sc64, e64 = dk.score_poses(0, poses, sd.SD_PREC_FP64)
        sc32, e32 = dk.score_poses(0, poses, sd.SD_PREC_MIXED)
    floor = np.maximum(np.abs(ref), 1.0)
    assert (np.abs(e64 - ref) / floor).max() < 1e-10
    assert (np.abs(e32 - ref) / floor).max() < 1e-5
    assert np.array_equal(sc64, -e64)


def test_pydock_gradients(cx, tables):
    osys = OracleSystem(cx, tables, scoring=1)
    ng = 6 + cx.n_modes_rec + cx.n_modes_lig
    poses = cx.poses.reshape(-1, cx.pose_len)[:12]
    with sd.Docking([cx], tables, scoring=sd.SD_SCORING_PYDOCK) as dk:
        e64, g64 = dk.pydock_grad(0, poses, sd.SD_PREC_FP64)
        e32, g32 = dk.pydock_grad(0, poses, sd.SD_PREC_MIXED)
    for k, pose in enumerate(poses):
        ref = oracle_grad(osys, pose, ng)
        scale = max(np.abs(ref).max(), 1.0)
        assert np.abs(g64[k] - ref).max() / scale < 1e-10
        assert np.abs(g32[k] - ref).max() / scale < 1e-4, (k, np.abs(g32[k] - ref).max() / scale)
        if k < 3:
            fd = fd_grad(osys, pose, ng)
            assert np.abs(g64[k] - fd).max() / scale < 1e-4  # FD truncation error is O(h^2)


def test_pydock_gso_step_locked(cx, tables):
    """GSO with pyDock scoring: mixed scores within 1e-5 of FP64, update bit-exact when fed them."""
    osys = OracleSystem(cx, tables, scoring=1)
    U = sd.gso_draws(3, cx.n_swarms, 4, cx.n_glowworms)
    st = OracleState(cx.n_swarms, cx.n_glowworms, cx.pose_len, cx.poses)
    with sd.Docking([cx], tables, scoring=sd.SD_SCORING_PYDOCK, precision=sd.SD_PREC_MIXED) as dk:
        for t in range(4):
            dk.set_state(0, sd.State(st.pos.copy(), st.scoring.copy(), st.luciferin.copy(), st.vision.copy(),
                                     st.step.copy(), st.moved.copy(), st.nnei.copy(), st.select.copy(),
                                     st.ref.copy()))
            dk.set_draws(0, U[:, t:t + 1, :])
            dk.step(1)
            g = dk.get_state(0)
            free = st.copy()
            oracle_step(osys, free, U[:, t, :])
            resc = (st.moved == 1) | (st.step == 0)
            err = np.abs(g.scoring[resc] - free.scoring[resc]) / np.maximum(np.abs(free.scoring[resc]), 1.0)
            assert err.size == 0 or err.max() <= 1e-5
            oracle_step(osys, st, U[:, t, :], score_override=g.scoring)
            assert np.array_equal(g.pos, st.pos) and np.array_equal(g.luciferin, st.luciferin)
