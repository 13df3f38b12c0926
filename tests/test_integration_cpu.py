"""The reference-side bindings (the C++ files a maintainer adds to the reference's build, kept in
sparkledock_b200/bindings/): they compile against the reference's own headers and this library's C
header, with warnings as errors for the bindings themselves; and the drop-in driver, the reference's
own prepare_gso_tasks compiled unmodified and linked to the hot-path binding and
libsparkle_b200.so, runs on a machine without a GPU up to the binding, which reports the missing
device instead of exiting."""
import os
import subprocess

import numpy as np
import pytest

from test_dropin import DROPIN, dropin_inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE = "/root/reference"
BINDINGS = [os.path.join(ROOT, "sparkledock_b200", "bindings", f) for f in ("cal_gso_tasks_b200.cc",
                                                                           "setup_b200.cc")]


@pytest.mark.parametrize("src", BINDINGS, ids=os.path.basename)
def test_reference_binding_compiles(src):
    if not os.path.isdir(os.path.join(REFERENCE, "source", "dock", "include")):
        pytest.skip("reference tree not present")
    inc = []
    for d in ("source/dock/include", "source/prep/include", "source/json/include"):
        inc += ["-isystem", os.path.join(REFERENCE, d)]  # the reference's headers: their warnings are not ours
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-Werror"] + inc +
                       ["-I", os.path.join(ROOT, "include"), src], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-3000:]


def test_dropin_driver_reaches_the_binding_without_gpu(tmp_path, tables):
    """Without a GPU the reference's prepare_gso_tasks still loads ./data/DCparams, types the atoms,
    computes the ellipsoid reference points and creates the swarm directories; then the binding's
    first C-ABI call fails with a status and a message (no exit), and the driver ends normally."""
    if not os.path.exists(DROPIN):
        pytest.skip("oracle/_ref/dropin_run not built (the reference sources are needed to build it)")
    import sparkledock_b200 as sd
    if sd.device_count() > 0:
        pytest.skip("a GPU is present: tests/test_dropin.py runs the whole path")
    args = dropin_inputs(tmp_path, tables, S=2, G=8)
    env = dict(os.environ, USE_CUDA="1", SPARKLE_STEPS="3", SPARKLE_PRECISION="fp64", NUM_THREADS="1")
    r = subprocess.run([DROPIN] + args, cwd=tmp_path, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "sparkle_b200: sd_ctx_create" in r.stderr
    assert (tmp_path / "swarm_0").is_dir() and (tmp_path / "swarm_1").is_dir()
    assert np.fromfile(tmp_path / "poses.bin").size == 2 * 8 * 27
