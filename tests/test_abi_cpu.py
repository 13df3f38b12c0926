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
