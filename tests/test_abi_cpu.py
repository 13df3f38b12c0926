"""The C-ABI library loads without a GPU and exports every function include/*.h declares;
host-only entry points (draws, synthetic systems) work on the CPU."""
import glob
import os
import re

import numpy as np

import sparkledock_b200 as sd
from sparkledock_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?\w+\s*\*?\s*(sd_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 20
    lib = _abi.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_abi.SIGNATURES), set(names) ^ set(_abi.SIGNATURES)


def test_version_and_device_count_without_gpu():
    assert b"sm_100a" in _abi.lib().sd_version()
    assert sd.device_count() >= 0


def test_synthetic_complex_properties():
    cx = sd.SyntheticComplex(757, 481, 5, 20, seed=4)
    for xyz, n in ((cx.rec_xyz, 757), (cx.lig_xyz, 481)):
        assert np.allclose(xyz.mean(0), 0, atol=1e-9)
        d2 = ((xyz[:, None, :] - xyz[None, :, :]) ** 2).sum(-1)
        d2[np.arange(n), np.arange(n)] = 1e9
        assert d2.min() >= 9.0 - 1e-9  # 3.0 A minimum separation
        assert np.sqrt((xyz ** 2).sum(1)).max() <= 2.2 * n ** (1 / 3) + 1.0
    M = cx.rec_modes.reshape(10, -1)
    assert np.allclose(M @ M.T, np.eye(10), atol=1e-10)
    assert set(np.unique(cx.rec_charge)) <= {-1.0, -0.5, 0.0, 0.5, 1.0}
    assert cx.rec_type.min() >= 0 and cx.rec_type.max() < 168
    q = cx.poses[..., 3:7]
    assert np.allclose((q ** 2).sum(-1), 1.0)
    again = sd.SyntheticComplex(757, 481, 5, 20, seed=4)
    assert np.array_equal(again.poses, cx.poses) and np.array_equal(again.rec_xyz, cx.rec_xyz)
    # the reference point is the descriptor's: assigning it changes what a context receives
    cx.lig_ref = [1.5, -2.0, 3.25]
    assert list(cx.desc.lig_ref_point) == [1.5, -2.0, 3.25] and np.array_equal(cx.lig_ref, [1.5, -2.0, 3.25])


def test_synthetic_arrays_outlive_their_complex():
    """An array taken from a temporary complex keeps the complex's buffer alive."""
    import gc
    keep = sd.SyntheticComplex(757, 481, 5, 20, seed=4)
    xyz, poses = sd.SyntheticComplex(757, 481, 5, 20, seed=4).lig_xyz, sd.SyntheticComplex(757, 481, 5, 20,
                                                                                            seed=4).poses
    gc.collect()
    junk = [np.full(1 << 20, np.nan) for _ in range(8)]  # reuse whatever memory was released
    assert np.array_equal(xyz, keep.lig_xyz) and np.array_equal(poses, keep.poses)
    del junk


def test_ctx_create_without_gpu_is_a_status_not_a_crash(tables):
    if sd.device_count() > 0:
        return
    cx = sd.SyntheticComplex(50, 40, 1, 8, seed=1)
    try:
        sd.Docking([cx], tables)
    except sd.SparkleError as e:
        assert e.code == _abi.SD_ERR_CUDA
    else:
        raise AssertionError("expected SD_ERR_CUDA without a device")


def test_gso_output_writer_format(tmp_path):
    """gso_<steps>.out matches the reference writer's line format (prepare_gso_task.cu:2850-2904)."""
    import ctypes as C
    S, G, pl = 2, 3, 27
    rng = np.random.default_rng(0)
    pos = rng.normal(size=(S, G, pl))
    luc = rng.normal(size=(S, G))
    nn = rng.integers(0, 6, size=(S, G)).astype(np.int32)
    vr = rng.uniform(0, 5, size=(S, G))
    sc = rng.normal(size=(S, G))
    rc = _abi.lib().sd_write_gso_output(str(tmp_path).encode(), 7, S, G, pl, 100, _abi.dptr(pos), _abi.dptr(luc),
                                        _abi.iptr(nn), _abi.dptr(vr), _abi.dptr(sc))
    assert rc == 0
    for s in range(S):
        lines = open(tmp_path / f"swarm_{7 + s}" / "gso_100.out").read().split("\n")
        assert lines[0] == "#Coordinates  RecID  LigID  Luciferin  Neighbor's number  Vision Range  Scoring"
        for g in range(G):
            exp = "(" + ", ".join("%f" % v for v in pos[s, g]) + ")\t0\t0\t" + "%f" % luc[s, g] + "\t" + \
                  str(nn[s, g]) + "\t" + "%f" % vr[s, g] + "\t" + "%f" % sc[s, g] + "\t"
            assert lines[1 + g] == exp


def test_forced_device_budget_gives_oom_status(tables, monkeypatch):
    """Fault injection on the host: a tiny forced device budget turns context creation into an
    SD_ERR_OOM status (no device is touched, so this runs without a GPU)."""
    monkeypatch.setenv("SPARKLE_DEVICE_BUDGET_MB", "1")
    cx = sd.SyntheticComplex(3002, 1274, 40, 200, seed=1)
    try:
        sd.Docking([cx], tables)
    except sd.SparkleError as e:
        assert e.code == _abi.SD_ERR_OOM
        assert "SPARKLE_DEVICE_BUDGET_MB" in str(e)
    else:
        raise AssertionError("expected SD_ERR_OOM")


def test_invalid_descriptors_are_rejected(tables):
    """Malformed inputs fail with SD_ERR_ARG / SD_ERR_NUMERIC before any device work."""
    cx = sd.SyntheticComplex(60, 40, 1, 8, seed=2)
    bad = sd.SyntheticComplex(60, 40, 1, 8, seed=2)
    bad.rec_type[3] = 168
    with __import__("pytest").raises(sd.SparkleError) as e:
        sd.Docking([bad], tables)
    assert e.value.code == _abi.SD_ERR_ARG
    nan = sd.SyntheticComplex(60, 40, 1, 8, seed=2)
    nan.lig_xyz[0, 0] = float("nan")
    with __import__("pytest").raises(sd.SparkleError) as e:
        sd.Docking([nan], tables)
    assert e.value.code == _abi.SD_ERR_NUMERIC
    t2 = (tables[0].copy(), tables[1], tables[2])
    t2[0][5] = float("inf")
    if sd.device_count() > 0:
        with __import__("pytest").raises(sd.SparkleError) as e:
            sd.Docking([cx], t2)
        assert e.value.code == _abi.SD_ERR_NUMERIC
