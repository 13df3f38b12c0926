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


def test_refinement_never_raises_fp64_energy(cx, tables):
    """sd_refine_poses: FP64 energies non-increasing, reported energies equal a fresh FP64 score
    (within 1e-10: the FP64 pyDock kernel's sum order follows its dynamic tile scheduling)."""
    poses = cx.poses.reshape(-1, cx.pose_len)[:16]
    with sd.Docking([cx], tables, scoring=sd.SD_SCORING_PYDOCK) as dk:
        p1, e0, e1 = dk.refine(0, poses, iters=20, step=0.5)
        _, e_check = dk.score_poses(0, p1, sd.SD_PREC_FP64)
    assert np.all(e1 <= e0)
    assert np.allclose(e1, e_check, rtol=1e-10, atol=1e-10)
    assert (e0 - e1).mean() > 0.0


def make_energy_fn(dk, base, precision):
    """torch.autograd.Function over the C ABI (test harness only): E(delta) for pose increments
    delta = (dt, dw, de) applied to fixed base poses (rotation q <- exp(dw/2) q), with the
    gradient from sd_pydock_grad."""
    import torch
    from pydock_util import qmul

    def apply(base_pose, d):
        p = np.array(base_pose, np.float64)
        p[:3] += d[:3]
        w = d[3:6]
        th = np.linalg.norm(w)
        if th > 0:
            dq = np.array([np.cos(th / 2), *(np.sin(th / 2) * w / th)])
            p[3:7] = qmul(dq, p[3:7])
        p[7:] += d[6:]
        return p

    class Fn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, delta):
            poses = np.stack([apply(b, d) for b, d in zip(base, delta.detach().cpu().numpy())])
            e, g = dk.pydock_grad(0, poses, precision)
            ctx.save_for_backward(torch.from_numpy(g))
            return torch.from_numpy(e)

        @staticmethod
        def backward(ctx, gout):
            (g,) = ctx.saved_tensors
            return gout[:, None] * g

    return Fn


def test_autograd_wrapper_gradcheck(cx, tables):
    import torch
    base = cx.poses.reshape(-1, cx.pose_len)[:3]
    ng = 6 + cx.n_modes_rec + cx.n_modes_lig
    with sd.Docking([cx], tables, scoring=sd.SD_SCORING_PYDOCK) as dk:
        Fn = make_energy_fn(dk, base, sd.SD_PREC_FP64)
        delta = torch.zeros((3, ng), dtype=torch.float64, requires_grad=True)
        # central differences (h = 1e-4, FP64) against the adjoint; the differences carry O(h^2)
        assert torch.autograd.gradcheck(Fn.apply, (delta,), eps=1e-4, atol=1e-2, rtol=1e-4)
        # the FP32 adjoint through the same wrapper matches the FP64 gradient within 1e-4
        Fn32 = make_energy_fn(dk, base, sd.SD_PREC_MIXED)
        d32 = torch.zeros((3, ng), dtype=torch.float64, requires_grad=True)
        Fn32.apply(d32).sum().backward()
        d64 = torch.zeros((3, ng), dtype=torch.float64, requires_grad=True)
        Fn.apply(d64).sum().backward()
        scale = d64.grad.abs().max(dim=1, keepdim=True).values.clamp(min=1.0)
        assert ((d32.grad - d64.grad).abs() / scale).max() < 1e-4
