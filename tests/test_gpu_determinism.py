"""Run-to-run reproducibility of the mixed-precision path and the device arithmetic of the slerp.

* The mixed DFIRE kernel sums each receptor tile's pairs in an order fixed by the pose and the tile
  and adds the tiles in tile order, so two runs from the same seed give the same bits in every
  state field for 100 GSO steps (single complex of the first benchmark configuration's size),
  whichever compiled variant runs; and every variant, the GSO step and the stateless scoring call
  give identical energies for the same poses.
* The correctly rounded acos and sin that the slerp of the GSO update uses
  (prepare_gso_tasks.cc:1370-1421) are evaluated on the device over 3.2 million points of the
  slerp's domain and compared bit for bit with the oracle's host restatement, which the CPU tests
  pin against mpmath."""
import ctypes as C

import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import _d, oracle
from sparkledock_b200 import _abi

pytestmark = pytest.mark.gpu
FIELDS = ("pos", "scoring", "luciferin", "vision_range", "step", "moved", "nnei_len", "select",
          "ligand_reference_pose")


def run_mixed(cx, tables, U, steps, variant, monkeypatch):
    monkeypatch.setenv("SPARKLE_MIXED_VARIANT", str(variant))
    with sd.Docking([cx], tables, precision=sd.SD_PREC_MIXED) as dk:
        dk.init_state(0, cx.poses)
        dk.set_draws(0, U)
        dk.step(steps)
        assert dk.tuning()["variant"] == variant
        return dk.get_state(0)


def test_two_mixed_runs_bit_identical(tables, monkeypatch):
    cx = sd.SyntheticComplex(757, 481, 130, 200, 10, 10, seed=100)
    steps = 100
    U = sd.gso_draws(0, cx.n_swarms, steps, cx.n_glowworms)
    a = run_mixed(cx, tables, U, steps, 0, monkeypatch)
    b = run_mixed(cx, tables, U, steps, 0, monkeypatch)
    c = run_mixed(cx, tables, U, steps, sd.mixed_variant_count() - 1, monkeypatch)
    for f in FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f"{f}: two runs differ"
        assert np.array_equal(getattr(a, f), getattr(c, f)), f"{f}: variants differ"


def test_variants_and_entry_points_give_identical_energies(tables, monkeypatch):
    cx = sd.SyntheticComplex(3002, 1274, 2, 200, 10, 10, seed=100)
    poses = cx.poses.reshape(-1, cx.pose_len)
    first = None
    for v in range(sd.mixed_variant_count()):
        monkeypatch.setenv("SPARKLE_MIXED_VARIANT", str(v))
        with sd.Docking([cx], tables, precision=sd.SD_PREC_MIXED) as dk:
            dk.init_state(0, cx.poses)
            dk.set_draws(0, sd.gso_draws(0, cx.n_swarms, 1, cx.n_glowworms))
            dk.step(1)  # step 0 scores every pose with the forced variant
            assert dk.tuning()["variant"] == v
            step_scores = dk.get_state(0).scoring.ravel()
            sc, en = dk.score_poses(0, poses, sd.SD_PREC_MIXED)
            assert np.array_equal(sc, step_scores), f"variant {v}: GSO step and stateless scores differ"
            if first is None:
                first = en
            assert np.array_equal(en, first), f"variant {v}: energies differ from variant 0"


def slerp_domain(n, seed=3):
    """Points where the slerp evaluates acos (the dot product after the sign flip, [0, 0.9995])
    and sin (omega = acos(dot) and omega / 2), plus the whole of [-1, 1] for acos."""
    rng = np.random.default_rng(seed)
    dots = np.concatenate([rng.uniform(0.0, 0.9995, n), rng.uniform(-1.0, 1.0, n // 4),
                           np.linspace(0.0, 0.9995, n // 4)])
    omega = np.arccos(np.clip(dots[dots >= 0], 0.0, 0.9995))
    angles = np.concatenate([omega, 0.5 * omega, rng.uniform(0.0, 2.0, n // 4)])
    return dots, angles


def test_device_crmath_matches_oracle():
    dots, angles = slerp_domain(1_000_000)
    assert dots.size + angles.size >= 3_200_000
    for fn, x in ((0, dots), (1, angles)):
        x = np.ascontiguousarray(x)
        dev = np.empty_like(x)
        host = np.empty_like(x)
        rc = _abi.lib().sd_crmath_eval(0, fn, _abi.dptr(x), x.size, _abi.dptr(dev))
        assert rc == 0, _abi.lib().sd_last_error()
        oracle().or_crmath_eval(fn, _d(x), x.size, _d(host))
        bad = np.flatnonzero(dev != host)
        assert bad.size == 0, f"fn {fn}: {bad.size} of {x.size} differ, e.g. x={x[bad[:3]]}"
