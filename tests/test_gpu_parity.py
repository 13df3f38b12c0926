"""GPU parity of the DFIRE GSO path against the oracle, through the C ABI.

Bars (written in the tests):
  * FP64 modes: scores, energies, GSO state and every bin bit-identical to the oracle;
  * MIXED: every bin bit-identical, |E_gpu - E_64| / max(|E_64|, 1) <= 1e-5 per pose, and the
    GSO update bit-identical when fed the GPU's own scores (step-locked, every step).
"""
import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import OracleState, OracleSystem, oracle_bins, oracle_cluster, oracle_scores, oracle_step

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-5
STATE_FIELDS = (("pos", "pos"), ("scoring", "scoring"), ("luciferin", "luciferin"),
                ("vision_range", "vision"), ("step", "step"), ("moved", "moved"), ("nnei_len", "nnei"),
                ("select", "select"), ("ligand_reference_pose", "ref"))


def rel_err(a, b, floor=1.0):
    return np.abs(np.asarray(a) - np.asarray(b)) / np.maximum(np.abs(b), floor)


@pytest.fixture(scope="module")
def c0():
    # config-0 atom counts, few swarms so the oracle finishes in seconds
    return sd.SyntheticComplex(757, 481, 3, 200, seed=7)


def test_scores_all_precisions(c0, tables):
    osys = OracleSystem(c0, tables)
    poses = c0.poses.reshape(-1, c0.pose_len)[:240]
    ref_sc, ref_en = oracle_scores(osys, poses)
    with sd.Docking([c0], tables) as dk:
        for prec in (sd.SD_PREC_FP64_REF, sd.SD_PREC_FP64):
            sc, en = dk.score_poses(0, poses, prec)
            assert np.array_equal(en, ref_en), f"precision {prec}: FP64 energies not bit-identical"
            assert np.array_equal(sc, ref_sc)
        sc, en = dk.score_poses(0, poses, sd.SD_PREC_MIXED)
        assert rel_err(en, ref_en).max() <= MIXED_TOL
        assert rel_err(sc, ref_sc).max() <= MIXED_TOL


def test_bins_bit_exact(c0, tables):
    osys = OracleSystem(c0, tables)
    poses = c0.poses.reshape(-1, c0.pose_len)
    with sd.Docking([c0], tables) as dk:
        for k in (0, 17, 333):
            ob, _, _, _, _ = oracle_bins(osys, poses[k])
            assert (ob >= 0).sum() > 0
            for prec in (sd.SD_PREC_FP64, sd.SD_PREC_MIXED):
                gb = dk.dfire_bins(0, poses[k], prec)
                assert np.array_equal(gb, ob), f"pose {k} precision {prec}: bins differ"


def test_gso_trajectory_fp64_bit_exact(c0, tables):
    steps = 25
    U = sd.gso_draws(0, c0.n_swarms, steps, c0.n_glowworms)
    osys = OracleSystem(c0, tables)
    st = OracleState(c0.n_swarms, c0.n_glowworms, c0.pose_len, c0.poses)
    with sd.Docking([c0], tables, precision=sd.SD_PREC_FP64) as dk:
        dk.init_state(0, c0.poses)
        dk.set_draws(0, U)
        for t in range(steps):
            oracle_step(osys, st, U[:, t, :])
            dk.step(1)
            g = dk.get_state(0)
            for f, o in STATE_FIELDS:
                assert np.array_equal(getattr(g, f), getattr(st, o)), f"step {t}: {f} differs"
        stats = dk.stats()
    assert stats["steps"] == steps
    assert stats["edge_u_zero"] == 0 and stats["edge_shortfall"] == 0


@pytest.mark.parametrize("precision", [sd.SD_PREC_FP64, sd.SD_PREC_MIXED])
def test_gso_without_modes(precision, tables):
    """A run without ANM (use_anm false: 0 + 0 modes, 7-element poses): FP64 state bit-identical to
    the oracle's every step; mixed scores within the bar and its GSO update bit-identical when fed
    the GPU's own scores."""
    cx = sd.SyntheticComplex(757, 481, 2, 100, n_modes_rec=0, n_modes_lig=0, seed=91)
    assert cx.pose_len == 7
    steps = 10
    U = sd.gso_draws(3, cx.n_swarms, steps, cx.n_glowworms)
    osys = OracleSystem(cx, tables)
    st = OracleState(cx.n_swarms, cx.n_glowworms, cx.pose_len, cx.poses)
    with sd.Docking([cx], tables, precision=precision) as dk:
        dk.init_state(0, cx.poses)
        dk.set_draws(0, U)
        for t in range(steps):
            if precision == sd.SD_PREC_FP64:
                oracle_step(osys, st, U[:, t, :])
                dk.step(1)
                g = dk.get_state(0)
            else:
                rescored = (st.moved == 1) | (st.step == 0)
                free = st.copy()
                oracle_step(osys, free, U[:, t, :])
                dk.step(1)
                g = dk.get_state(0)
                if rescored.any():
                    assert rel_err(g.scoring[rescored], free.scoring[rescored]).max() <= MIXED_TOL
                oracle_step(osys, st, U[:, t, :], score_override=g.scoring)
            for f, o in STATE_FIELDS:
                assert np.array_equal(getattr(g, f), getattr(st, o)), f"step {t}: {f} differs"


def test_gso_step_locked_mixed(c0, tables):
    steps = 12
    U = sd.gso_draws(1, c0.n_swarms, steps, c0.n_glowworms)
    osys = OracleSystem(c0, tables)
    st = OracleState(c0.n_swarms, c0.n_glowworms, c0.pose_len, c0.poses)
    worst = 0.0
    with sd.Docking([c0], tables, precision=sd.SD_PREC_MIXED) as dk:
        for t in range(steps):
            gs = sd.State(st.pos.copy(), st.scoring.copy(), st.luciferin.copy(), st.vision.copy(),
                          st.step.copy(), st.moved.copy(), st.nnei.copy(), st.select.copy(), st.ref.copy())
            dk.set_state(0, gs)
            dk.set_draws(0, U[:, t:t + 1, :])
            dk.step(1)
            g = dk.get_state(0)
            rescored = (st.moved == 1) | (st.step == 0)
            # FP64 oracle energies of the rescored poses at the pre-step state
            free = st.copy()
            oracle_step(osys, free, U[:, t, :])
            err = rel_err(g.scoring[rescored], free.scoring[rescored])
            worst = max(worst, float(err.max()) if err.size else 0.0)
            assert worst <= MIXED_TOL, f"step {t}: score error {worst:.3g}"
            # the GSO update fed with the GPU's scores must be bit-identical
            oracle_step(osys, st, U[:, t, :], score_override=g.scoring)
            for f, o in STATE_FIELDS:
                assert np.array_equal(getattr(g, f), getattr(st, o)), f"step {t}: {f} differs"


def test_multi_complex_batch_fp64(tables):
    cxs = [sd.SyntheticComplex(300, 200, 2, 50, seed=21), sd.SyntheticComplex(520, 140, 3, 32, seed=22),
           sd.SyntheticComplex(180, 260, 1, 96, n_modes_rec=4, n_modes_lig=0, seed=23)]
    steps = 6
    Us = [sd.gso_draws(5 + i, c.n_swarms, steps, c.n_glowworms) for i, c in enumerate(cxs)]
    osyss = [OracleSystem(c, tables) for c in cxs]
    sts = [OracleState(c.n_swarms, c.n_glowworms, c.pose_len, c.poses) for c in cxs]
    with sd.Docking(cxs, tables, precision=sd.SD_PREC_FP64) as dk:
        for i, c in enumerate(cxs):
            dk.init_state(i, c.poses)
            dk.set_draws(i, Us[i])
        for t in range(steps):
            dk.step(1)
            for i in range(len(cxs)):
                oracle_step(osyss[i], sts[i], Us[i][:, t, :])
                g = dk.get_state(i)
                for f, o in STATE_FIELDS:
                    assert np.array_equal(getattr(g, f), getattr(sts[i], o)), f"complex {i} step {t}: {f}"


def test_errors_are_status_codes(c0, tables):
    with sd.Docking([c0], tables) as dk:
        with pytest.raises(sd.SparkleError) as e:
            dk.step(1)  # no state yet
        assert e.value.code == 6
        dk.init_state(0, c0.poses)
        with pytest.raises(sd.SparkleError) as e:
            dk.step(1)  # no draws yet
        assert e.value.code == 6
        bad = c0.poses.copy()
        bad[0, 0, 0] = np.nan
        with pytest.raises(sd.SparkleError) as e:
            dk.score_poses(0, bad.reshape(-1, c0.pose_len)[:2])
        assert e.value.code == 5


def test_multi_complex_batch_mixed_scores(tables):
    """Batched complexes of uneven sizes in one persistent launch (mixed): every rescored pose
    of one GSO step within 1e-5 of the FP64 oracle."""
    cxs = [sd.SyntheticComplex(757, 481, 2, 40, seed=51), sd.SyntheticComplex(2039, 1440, 1, 40, seed=52),
           sd.SyntheticComplex(6143, 633, 1, 40, seed=53)]
    with sd.Docking(cxs, tables, precision=sd.SD_PREC_MIXED) as dk:
        for i, c in enumerate(cxs):
            dk.init_state(i, c.poses)
            dk.set_draws(i, sd.gso_draws(9 + i, c.n_swarms, 1, c.n_glowworms))
        dk.step(1)
        for i, c in enumerate(cxs):
            g = dk.get_state(i)
            ref_sc, _ = oracle_scores(OracleSystem(c, tables), c.poses)
            assert rel_err(g.scoring.ravel(), ref_sc).max() <= MIXED_TOL, f"complex {i}"


@pytest.mark.parametrize("variant", range(sd.mixed_variant_count()))
def test_every_mixed_kernel_variant(variant, c0, tables, monkeypatch):
    """Each compiled variant of the mixed kernel (the autotuner may pick any) scores the first
    step's poses within 1e-5 of the FP64 oracle, with no index guard firing."""
    monkeypatch.setenv("SPARKLE_MIXED_VARIANT", str(variant))
    osys = OracleSystem(c0, tables)
    ref_sc, _ = oracle_scores(osys, c0.poses)
    with sd.Docking([c0], tables, precision=sd.SD_PREC_MIXED) as dk:
        dk.init_state(0, c0.poses)
        dk.set_draws(0, sd.gso_draws(0, c0.n_swarms, 1, c0.n_glowworms))
        dk.step(1)
        assert dk.tuning()["variant"] == variant
        g = dk.get_state(0)
        assert rel_err(g.scoring.ravel(), ref_sc).max() <= MIXED_TOL
        st = dk.stats()
        assert st["pairs_in_cutoff"] > 0


def _edge_sweep_complex():
    """One receptor atom at the origin and one ligand atom at the ligand-frame origin; every other
    atom more than 100 A away, so each pose has exactly one candidate pair, at distance |t|."""
    cx = sd.SyntheticComplex(40, 30, 1, 4, n_modes_rec=0, n_modes_lig=0, seed=3)
    for i in range(cx.n_rec):
        cx.rec_xyz[i] = (-100.0 - 3.0 * i, 0.0, 0.0)
    for j in range(cx.n_lig):
        cx.lig_xyz[j] = (100.0 + 3.0 * j, 0.0, 0.0)
    cx.rec_xyz[0] = (0.0, 0.0, 0.0)
    cx.lig_xyz[0] = (0.0, 0.0, 0.0)
    d = [np.sqrt(((k + 1) / 2.0) ** 2) * (1.0 + m * 1e-7) for k in range(1, 30) for m in range(-60, 61, 4)]
    d += [15.0 + m * 1e-6 for m in range(-150, 151, 3)]
    d += [0.05 * m for m in range(1, 12)]
    poses = np.zeros((len(d), cx.pose_len))
    poses[:, 0] = d
    poses[:, 3] = 1.0
    return cx, np.concatenate([poses, _cutoff_window_poses(cx)])


def _cutoff_window_poses(cx):
    """Poses whose FP32 pair distance lands exactly on the mixed kernel's FP32 cutoff
    cut2 = 225 + B and on its neighbouring floats (B, the FP32 error bound, evaluated in the
    kernel's operation order).  d2 = fma(ey, ey, ex * ex) for the pair (rec atom 0 at the origin,
    ligand atom 0 at t, coordinates centred on t)."""
    f = np.float32
    lr = float(np.sqrt((cx.lig_xyz ** 2).sum(1)).max()) * (1 + 1e-6) + 1e-4
    lig_radius = f(lr)
    if float(lig_radius) < lr:
        lig_radius = np.nextafter(lig_radius, f(np.inf))
    u = f(5.9604645e-8)
    RL = f(lig_radius + f(1e-4))                 # dL = 0 * 1.0001 + 1e-4 without modes
    t4 = f(f(f(26.2) * f(f(f(2.0) * RL) + f(15.1))) + f(228.0))
    B = f(f(f(2.0) * f(f(f(f(2.02) * u) * t4) + f(f(f(3.0) * u) * f(228.0)))) + f(1e-6))
    cut2 = f(f(225.0) + B)
    targets = {float(cut2)}
    x = cut2
    for _ in range(3):
        x = np.nextafter(x, f(np.inf)); targets.add(float(x))
    x = cut2
    for _ in range(3):
        x = np.nextafter(x, f(0)); targets.add(float(x))
    out = []
    tx0 = f(np.sqrt(np.float64(cut2)))
    for k in range(-40, 41):
        ex = f(tx0 + f(k) * f(9.5367432e-07))
        p = f(np.float64(ex) * np.float64(ex))
        for ey in (0.0, 1e-3, 2e-3, 3e-3, 4e-3, 6e-3, 8e-3, 1.1e-2):
            ey = f(ey)
            d2 = f(np.float64(ey) * np.float64(ey) + np.float64(p))
            if float(d2) in targets:
                pose = np.zeros(cx.pose_len)
                pose[0], pose[1], pose[3] = -float(ex), -float(ey), 1.0
                out.append(pose)
                targets.discard(float(d2))
    assert float(cut2) not in targets, "no pose lands on the FP32 cutoff"
    return np.array(out)


@pytest.mark.parametrize("variant", range(sd.mixed_variant_count()))
def test_single_pair_sweep_across_bin_edges(variant, tables, monkeypatch):
    """A single pair swept across every DFIRE bin edge and across the cutoff within the FP32 error
    bound: each compiled mixed variant gives the oracle's energy for every distance (a wrong bin or
    a pair counted past the cutoff shows up as an O(1) error), and FP64 is bit-identical."""
    monkeypatch.setenv("SPARKLE_MIXED_VARIANT", str(variant))
    cx, poses = _edge_sweep_complex()
    _, ref_en = oracle_scores(OracleSystem(cx, tables), poses)
    with sd.Docking([cx], tables, precision=sd.SD_PREC_MIXED) as dk:
        dk.init_state(0, np.tile(poses[:1], (cx.n_swarms * cx.n_glowworms, 1)).reshape(cx.poses.shape))
        dk.set_draws(0, sd.gso_draws(0, cx.n_swarms, 1, cx.n_glowworms))
        dk.step(1)  # selects the forced variant
        assert dk.tuning()["variant"] == variant
        _, en = dk.score_poses(0, poses, sd.SD_PREC_MIXED)
        assert np.abs(en - ref_en).max() <= 1e-12, np.nonzero(np.abs(en - ref_en) > 1e-12)
        _, en64 = dk.score_poses(0, poses, sd.SD_PREC_FP64)
        assert np.array_equal(en64, ref_en)
        assert dk.stats()["pairs_fallback"] > 0


@pytest.mark.parametrize("variant", range(sd.mixed_variant_count()))
def test_large_anm_extents_loose_tiles(variant, tables, monkeypatch):
    """Poses with ANM extents large enough that the displacement bound makes the FP16 stage-1
    error bound too wide (tile bound R > 40 A): those tiles pass every candidate and stage 2
    filters exactly; energies still match the FP64 oracle, and FP64 stays bit-identical."""
    monkeypatch.setenv("SPARKLE_MIXED_VARIANT", str(variant))
    cx = sd.SyntheticComplex(757, 481, 1, 64, seed=61)
    poses = cx.poses.reshape(-1, cx.pose_len).copy()[:64]
    rng = np.random.default_rng(5)
    poses[:, 7:] *= rng.uniform(1.0, 150.0, size=(len(poses), 1))  # displacement bounds up to ~120 A
    _, ref_en = oracle_scores(OracleSystem(cx, tables), poses)
    with sd.Docking([cx], tables, precision=sd.SD_PREC_MIXED) as dk:
        dk.init_state(0, cx.poses)
        dk.set_draws(0, sd.gso_draws(0, cx.n_swarms, 1, cx.n_glowworms))
        dk.step(1)
        assert dk.tuning()["variant"] == variant
        _, en = dk.score_poses(0, poses, sd.SD_PREC_MIXED)
        assert rel_err(en, ref_en).max() <= MIXED_TOL
        _, en64 = dk.score_poses(0, poses, sd.SD_PREC_FP64)
        assert np.array_equal(en64, ref_en)


@pytest.mark.parametrize("precision", [sd.SD_PREC_FP64, sd.SD_PREC_MIXED])
def test_cluster_final_poses_match_oracle(precision, tables):
    """BSAS clustering of the final poses after GSO steps (sd_cluster) equals the oracle's on the
    same state: cluster count, representatives, sizes and every glowworm's cluster."""
    cx = sd.SyntheticComplex(757, 481, 3, 96, seed=71)
    rb = (np.arange(cx.n_rec) % 8 == 1).astype(np.int32)  # a backbone-like subset
    lb = (np.arange(cx.n_lig) % 8 == 1).astype(np.int32)
    with sd.Docking([cx], tables, precision=precision) as dk:
        dk.init_state(0, cx.poses)
        dk.set_draws(0, sd.gso_draws(4, cx.n_swarms, 10, cx.n_glowworms))
        dk.step(10)
        st = dk.get_state(0)
        got = dk.cluster(0, rb, lb)
    ref = oracle_cluster(OracleSystem(cx, tables), st.pos, st.scoring, rb, lb)
    assert np.array_equal(got["n_clusters"], ref["n_clusters"])
    for s in range(cx.n_swarms):
        n = ref["n_clusters"][s]
        assert np.array_equal(got["rep"][s, :n], ref["rep"][s, :n])
        assert np.array_equal(got["size"][s, :n], ref["size"][s, :n])
    assert np.array_equal(got["member"], ref["member"])
    # the first glowworm in score order is counted twice in cluster 0, as in the reference
    assert (ref["size"].sum(axis=1) == cx.n_glowworms + 1).all()
    assert 1 < ref["n_clusters"].min()
