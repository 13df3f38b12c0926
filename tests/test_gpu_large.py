"""Complexes larger than a CTA's shared memory, through the C ABI.

When the per-pose arrays of a scorer (transformed ligand atoms, per-receptor-atom FP64 partials,
tile lists) do not fit in the shared memory a CTA may use, the context switches that scorer to an
instantiation which keeps them in a per-CTA global scratch; the arithmetic, and so every bit of
the result, is unchanged.  Checked here:
  * receptor 30,000 / ligand 8,000 atoms (the FP64 scorers spill: ~620 KB per pose): FP64 energies
    bit-identical to the oracle, mixed within 1e-5 of them, a GSO step bit-identical, the pyDock
    adjoint (which spills too) within 1e-10 (FP64) of the oracle's gradient;
  * receptor 3,000 / ligand 20,000 atoms (every scorer spills, the mixed one included): the same
    bars, and the no-allocation scoring call refuses such a complex until an allocating call has
    sized the context's scratch, then matches the allocating call bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import OracleState, OracleSystem, oracle_scores, oracle_step
from pydock_util import oracle_grad
from sparkledock_b200 import _abi

pytestmark = pytest.mark.gpu
FIELDS = (("pos", "pos"), ("scoring", "scoring"), ("luciferin", "luciferin"), ("vision_range", "vision"),
          ("nnei_len", "nnei"), ("select", "select"), ("ligand_reference_pose", "ref"))


def rel_err(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)) / np.maximum(np.abs(b), 1.0)


@pytest.mark.parametrize("nr,nl", [(30000, 8000), (3000, 20000)])
def test_large_complex_scores_and_step(nr, nl, tables):
    cx = sd.SyntheticComplex(nr, nl, 1, 6, 10, 10, seed=31)
    poses = cx.poses.reshape(-1, cx.pose_len)
    ref_sc, ref_en = oracle_scores(OracleSystem(cx, tables), poses)
    with sd.Docking([cx], tables, precision=sd.SD_PREC_FP64) as dk:
        for prec in (sd.SD_PREC_FP64, sd.SD_PREC_FP64_REF):
            sc, en = dk.score_poses(0, poses, prec)
            assert np.array_equal(en, ref_en) and np.array_equal(sc, ref_sc), f"precision {prec}"
        _, e32 = dk.score_poses(0, poses, sd.SD_PREC_MIXED)
        assert rel_err(e32, ref_en).max() <= 1e-5
        U = sd.gso_draws(4, 1, 2, 6)
        dk.init_state(0, cx.poses)
        dk.set_draws(0, U)
        st = OracleState(1, 6, cx.pose_len, cx.poses)
        osys = OracleSystem(cx, tables)
        for t in range(2):
            dk.step(1)
            oracle_step(osys, st, U[:, t, :])
            g = dk.get_state(0)
            for f, o in FIELDS:
                assert np.array_equal(getattr(g, f), getattr(st, o)), f"step {t}: {f}"


def test_large_ligand_adjoint(tables):
    cx = sd.SyntheticComplex(3000, 8000, 1, 2, 10, 10, seed=32)
    poses = cx.poses.reshape(-1, cx.pose_len)
    ng = 6 + cx.n_modes_rec + cx.n_modes_lig
    with sd.Docking([cx], tables, scoring=sd.SD_SCORING_PYDOCK) as dk:
        _, g64 = dk.pydock_grad(0, poses, sd.SD_PREC_FP64)
        _, g32 = dk.pydock_grad(0, poses, sd.SD_PREC_MIXED)
    osys = OracleSystem(cx, tables, scoring=1)
    for k in range(len(poses)):
        ref = oracle_grad(osys, poses[k], ng)
        scale = max(np.abs(ref).max(), 1.0)
        assert np.abs(g64[k] - ref).max() / scale < 1e-10
        assert np.abs(g32[k] - ref).max() / scale < 1e-4


def test_noalloc_needs_a_sized_scratch_for_large_complexes(tables):
    import torch
    cx = sd.SyntheticComplex(3000, 20000, 1, 4, 10, 10, seed=33)
    poses = np.ascontiguousarray(cx.poses.reshape(-1, cx.pose_len))
    n = poses.shape[0]
    with sd.Docking([cx], tables) as dk:
        d_pose = torch.from_numpy(poses).cuda()
        d_sc = torch.empty(n, dtype=torch.float64, device="cuda")
        d_en = torch.empty(n, dtype=torch.float64, device="cuda")
        d_ref = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()

        def call():
            return _abi.lib().sd_score_poses_noalloc(dk._ctx, 0, C.c_void_p(d_pose.data_ptr()), n, sd.SD_PREC_MIXED,
                                                     C.c_void_p(d_sc.data_ptr()), C.c_void_p(d_en.data_ptr()),
                                                     C.c_void_p(d_ref.data_ptr()), 1)
        assert call() == _abi.SD_ERR_NOTSUP and b"global scratch" in _abi.lib().sd_last_error()
        sc, en = dk.score_poses(0, poses, sd.SD_PREC_MIXED)  # sizes the context's scratch
        assert call() == 0, _abi.lib().sd_last_error()
        assert np.array_equal(d_sc.cpu().numpy(), sc) and np.array_equal(d_en.cpu().numpy(), en)


@pytest.mark.parametrize("precision", [sd.SD_PREC_FP64, sd.SD_PREC_MIXED], ids=["fp64", "mixed"])
def test_swarms_larger_than_a_cta(precision, tables):
    """Swarms of more than 1,024 glowworms (one CTA's threads) next to an ordinary one in the same
    context: every state field bit-identical to the oracle every step (FP64), or when the oracle's
    update is fed the GPU's scores (mixed, step-locked)."""
    cxs = [sd.SyntheticComplex(300, 200, 2, 1500, 10, 10, seed=34), sd.SyntheticComplex(400, 150, 1, 200, 10, 10,
                                                                                         seed=35)]
    steps = 3
    Us = [sd.gso_draws(6 + i, c.n_swarms, steps, c.n_glowworms) for i, c in enumerate(cxs)]
    osyss = [OracleSystem(c, tables) for c in cxs]
    sts = [OracleState(c.n_swarms, c.n_glowworms, c.pose_len, c.poses) for c in cxs]
    with sd.Docking(cxs, tables, precision=precision) as dk:
        for i, c in enumerate(cxs):
            dk.init_state(i, c.poses)
            dk.set_draws(i, Us[i])
        for t in range(steps):
            dk.step(1)
            for i, c in enumerate(cxs):
                g = dk.get_state(i)
                if precision == sd.SD_PREC_FP64:
                    oracle_step(osyss[i], sts[i], Us[i][:, t, :])
                else:
                    free = sts[i].copy()
                    rescored = (free.moved == 1) | (free.step == 0)
                    oracle_step(osyss[i], free, Us[i][:, t, :])
                    assert rel_err(g.scoring[rescored], free.scoring[rescored]).max() <= 1e-5
                    oracle_step(osyss[i], sts[i], Us[i][:, t, :], score_override=g.scoring)
                for f, o in FIELDS + (("moved", "moved"), ("step", "step")):
                    assert np.array_equal(getattr(g, f), getattr(sts[i], o)), f"complex {i} step {t}: {f}"
