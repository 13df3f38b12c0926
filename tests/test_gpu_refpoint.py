"""The ligand reference point computed on the GPU (sd_reference_point_device) is bit-identical to
the host computation (sd_reference_point, itself pinned bit-identical to the reference's own
minimum_volume_ellipsoid by the CPU tests) on point clouds of many shapes and sizes and on the
ligands of the benchmark workloads."""
import numpy as np
import pytest

import sparkledock_b200 as sd
from sparkledock_b200 import _abi

pytestmark = pytest.mark.gpu


def test_device_reference_point_equals_host():
    rng = np.random.default_rng(5)
    clouds = [np.ascontiguousarray(rng.normal(size=(int(rng.integers(4, 3000)), 3)) * rng.uniform(0.5, 30, 3) +
                                   rng.uniform(-50, 50, 3)) for _ in range(20)]
    clouds += [sd.SyntheticComplex(100, nl, 1, 1, seed=100 + i).lig_xyz
               for i, nl in enumerate((481, 1274, 1440, 1061, 1256, 1658, 1138, 1766, 633, 1125))]
    for pts in clouds:
        pts = np.ascontiguousarray(pts)
        h, d = np.empty(3), np.empty(3)
        assert _abi.lib().sd_reference_point(_abi.dptr(pts), len(pts), _abi.dptr(h)) == 0
        assert _abi.lib().sd_reference_point_device(0, _abi.dptr(pts), len(pts), _abi.dptr(d)) == 0, \
            _abi.lib().sd_last_error()
        assert np.array_equal(h, d), (len(pts), h - d)
