"""GPU parity at the benchmark workloads' own atom counts, through the C ABI.

The benchmark configurations are the single complex (receptor 3002 / ligand 1274 atoms), the
batched eight complexes (757/481 ... 6143/633), the large receptor (17,307 / 1,125) and the pyDock
adjoint on the single complex.  Each is generated exactly as the benchmark generates it (same
seeds), with a few swarms so that the CPU oracle finishes in seconds.  Bars:
  * FP64 energies and every DFIRE bin bit-identical to the oracle (16 poses per complex);
  * mixed energies within |E - E64| / max(|E64|, 1) <= 1e-5 of the plain FP64 kernel (itself
    pinned bit-identical to the oracle) on every pose of the sample, and mixed bins identical;
  * the single complex's GSO update bit-identical to the oracle's for 3 steps when fed the GPU's
    mixed scores (step-locked), and a batched FP64 step of all eight complexes bit-identical;
  * the adjoint (FP32) within 1e-4 of the FP64 GPU gradient, which is within 1e-10 of the oracle's;
    its FP32 energy within the same 1e-4 (the FP32 pair terms of ~60k pairs per pose: 4.3e-5 was
    measured at this size, where the DFIRE scorer's FP64 table sums reach 1e-13).
"""
import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import OracleState, OracleSystem, oracle_bins, oracle_scores, oracle_step
from pydock_util import oracle_grad

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-5
C1 = (3002, 1274)
C2 = [(757, 481), (2039, 1440), (2516, 1061), (2030, 1256), (3052, 1658), (6058, 1138), (6032, 1766), (6143, 633)]
C3 = (17307, 1125)
STATE_FIELDS = (("pos", "pos"), ("scoring", "scoring"), ("luciferin", "luciferin"),
                ("vision_range", "vision"), ("step", "step"), ("moved", "moved"), ("nnei_len", "nnei"),
                ("select", "select"), ("ligand_reference_pose", "ref"))


def rel_err(a, b, floor=1.0):
    return np.abs(np.asarray(a) - np.asarray(b)) / np.maximum(np.abs(b), floor)


def check_complex(dk, ci, cx, tables, n_oracle=16, bins_pose=True):
    """FP64 (both kernels) bit-identical to the oracle on n_oracle poses; mixed within the bar of
    the FP64 kernel on every pose of the complex; bins of one pose identical in FP64 and mixed."""
    poses = cx.poses.reshape(-1, cx.pose_len)
    osys = OracleSystem(cx, tables)
    sel = poses[np.linspace(0, len(poses) - 1, n_oracle).astype(int)]
    ref_sc, ref_en = oracle_scores(osys, sel)
    for prec in (sd.SD_PREC_FP64, sd.SD_PREC_FP64_REF):
        sc, en = dk.score_poses(ci, sel, prec)
        assert np.array_equal(en, ref_en) and np.array_equal(sc, ref_sc), f"complex {ci} precision {prec}"
    s64, e64 = dk.score_poses(ci, poses, sd.SD_PREC_FP64)
    s32, e32 = dk.score_poses(ci, poses, sd.SD_PREC_MIXED)
    assert rel_err(e32, e64).max() <= MIXED_TOL, f"complex {ci}: mixed energy error {rel_err(e32, e64).max():.3g}"
    assert rel_err(s32, s64).max() <= MIXED_TOL
    if bins_pose:
        want, _, _, _, _ = oracle_bins(osys, sel[0])
        assert (want >= 0).any()
        for prec in (sd.SD_PREC_FP64, sd.SD_PREC_MIXED):
            assert np.array_equal(dk.dfire_bins(ci, sel[0], prec), want), f"complex {ci} bins, precision {prec}"
    return float(rel_err(e32, e64).max())


def test_single_complex_shape(tables):
    cx = sd.SyntheticComplex(*C1, 5, 200, 10, 10, seed=100)  # the benchmark's single complex, 5 of 402 swarms
    with sd.Docking([cx], tables) as dk:
        check_complex(dk, 0, cx, tables)


def test_single_complex_step_locked_gso(tables):
    """Three GSO steps of the single complex in mixed precision: the oracle's update fed with the
    GPU's scores gives the GPU's state bit for bit, and those scores are within the bar of the
    oracle's own FP64 scores, every step."""
    cx = sd.SyntheticComplex(*C1, 4, 200, 10, 10, seed=100)
    steps = 3
    U = sd.gso_draws(0, cx.n_swarms, steps, cx.n_glowworms)
    osys = OracleSystem(cx, tables)
    st = OracleState(cx.n_swarms, cx.n_glowworms, cx.pose_len, cx.poses)
    with sd.Docking([cx], tables, precision=sd.SD_PREC_MIXED) as dk:
        dk.init_state(0, cx.poses)
        dk.set_draws(0, U)
        for t in range(steps):
            rescored = (st.moved == 1) | (st.step == 0)
            free = st.copy()
            oracle_step(osys, free, U[:, t, :])
            dk.step(1)
            g = dk.get_state(0)
            assert rel_err(g.scoring[rescored], free.scoring[rescored]).max() <= MIXED_TOL, f"step {t}"
            oracle_step(osys, st, U[:, t, :], score_override=g.scoring)
            for f, o in STATE_FIELDS:
                assert np.array_equal(getattr(g, f), getattr(st, o)), f"step {t}: {f} differs"


def test_batched_eight_complexes(tables):
    """All eight complexes of the batched workload in one context (one persistent scorer launch per
    call): per-complex parity, then one batched FP64 GSO step bit-identical to the oracle."""
    cxs = [sd.SyntheticComplex(nr, nl, 2, 64, 10, 10, seed=100 + i) for i, (nr, nl) in enumerate(C2)]
    U = [sd.gso_draws(i, c.n_swarms, 1, c.n_glowworms) for i, c in enumerate(cxs)]
    with sd.Docking(cxs, tables, precision=sd.SD_PREC_FP64) as dk:
        for i, c in enumerate(cxs):
            check_complex(dk, i, c, tables, n_oracle=8, bins_pose=i in (0, 7))
            dk.init_state(i, c.poses)
            dk.set_draws(i, U[i])
        dk.step(1)
        for i, c in enumerate(cxs):
            st = OracleState(c.n_swarms, c.n_glowworms, c.pose_len, c.poses)
            oracle_step(OracleSystem(c, tables), st, U[i][:, 0, :])
            g = dk.get_state(i)
            for f, o in STATE_FIELDS:
                assert np.array_equal(getattr(g, f), getattr(st, o)), f"complex {i}: {f} differs"


def test_large_receptor_shape(tables):
    cx = sd.SyntheticComplex(*C3, 2, 200, 10, 10, seed=100)  # the large-receptor workload, 2 of 1245 swarms
    with sd.Docking([cx], tables) as dk:
        check_complex(dk, 0, cx, tables, n_oracle=12)


def test_adjoint_shape(tables):
    """The pyDock-style adjoint on the single complex's atom counts: FP32 gradient within 1e-4 of the
    FP64 GPU gradient on 512 poses (max-norm relative per pose), FP64 within 1e-10 of the oracle's
    on 4 poses."""
    cx = sd.SyntheticComplex(*C1, 3, 200, 10, 10, seed=100)
    ng = 6 + cx.n_modes_rec + cx.n_modes_lig
    poses = cx.poses.reshape(-1, cx.pose_len)[:512]
    with sd.Docking([cx], tables, scoring=sd.SD_SCORING_PYDOCK) as dk:
        e64, g64 = dk.pydock_grad(0, poses, sd.SD_PREC_FP64)
        e32, g32 = dk.pydock_grad(0, poses, sd.SD_PREC_MIXED)
    scale = np.maximum(np.abs(g64).max(axis=1), 1.0)
    assert (np.abs(g32 - g64).max(axis=1) / scale).max() <= 1e-4
    assert rel_err(e32, e64).max() <= 1e-4
    osys = OracleSystem(cx, tables, scoring=1)
    for k in range(4):
        ref = oracle_grad(osys, poses[k], ng)
        assert np.abs(g64[k] - ref).max() / max(np.abs(ref).max(), 1.0) < 1e-10
