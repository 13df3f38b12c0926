"""Checkpoints of a GSO state (sd_write_checkpoint / sd_read_checkpoint).

CPU: a state survives the file bit for bit; other sizes, a truncated file, a corrupted byte and
a file that is not a checkpoint are refused; no partial file is left behind.
GPU: a run stopped after some steps, written to a checkpoint, read into a new context and given
the remaining draws ends in the same state, bit for bit, as the uninterrupted run (FP64); the
mixed path restores the saved state exactly and continues.
"""
import os

import numpy as np
import pytest

import sparkledock_b200 as sd

STATE_FIELDS = ("pos", "scoring", "luciferin", "vision_range", "step", "moved", "nnei_len", "select",
                "ligand_reference_pose")


def _random_state(S, G, pl, seed):
    rng = np.random.default_rng(seed)
    st = sd.State.empty(S, G, pl)
    for f in STATE_FIELDS:
        a = getattr(st, f)
        if a.dtype == np.int32:
            a[:] = rng.integers(-5, 1000, a.shape)
        else:
            a[:] = rng.normal(0, 50, a.shape)
    st.pos[0, 0, 0] = -0.0
    st.scoring[0, 1] = np.nextafter(0.0, 1.0)  # a subnormal survives too
    return st


def _equal(a, b):
    return all(np.array_equal(getattr(a, f), getattr(b, f)) and
               np.array_equal(np.signbit(getattr(a, f)), np.signbit(getattr(b, f))) for f in STATE_FIELDS)


def test_checkpoint_roundtrip(tmp_path):
    st = _random_state(3, 17, 27, 1)
    path = tmp_path / "run.ckpt"
    sd.write_checkpoint(path, st, 42, 100)
    back, steps, total = sd.read_checkpoint(path)
    assert steps == 42 and total == 100 and _equal(st, back)
    assert not os.path.exists(str(path) + ".partial")


def test_checkpoint_refuses_bad_files(tmp_path):
    st = _random_state(2, 5, 7, 2)
    path = tmp_path / "run.ckpt"
    sd.write_checkpoint(path, st, 3)
    raw = path.read_bytes()
    lib = sd._abi.lib()
    # other sizes than the file's
    other = sd.State.empty(2, 6, 7)
    cs = other.as_c()
    steps = sd.C.c_longlong()
    assert lib.sd_read_checkpoint(str(path).encode(), 2, 6, 7, sd.C.byref(steps), None, sd.C.byref(cs)) != 0
    assert "sizes" in sd._abi.lib().sd_last_error().decode()
    # truncated, corrupted, extended, foreign
    for name, data in (("trunc", raw[:-9]), ("flip", raw[:40] + bytes([raw[40] ^ 1]) + raw[41:]),
                       ("extra", raw + b"\0"), ("foreign", b"not a checkpoint at all" * 4)):
        bad = tmp_path / f"{name}.ckpt"
        bad.write_bytes(data)
        with pytest.raises(sd.SparkleError):
            sd.read_checkpoint(bad)
    with pytest.raises(sd.SparkleError):
        sd.read_checkpoint(tmp_path / "missing.ckpt")


@pytest.mark.gpu
def test_resume_from_checkpoint_is_bit_exact(tmp_path, tables):
    cx = sd.SyntheticComplex(757, 481, 3, 100, seed=81)
    steps, stop = 10, 4
    U = sd.gso_draws(5, cx.n_swarms, steps, cx.n_glowworms)
    with sd.Docking([cx], tables, precision=sd.SD_PREC_FP64) as dk:
        dk.init_state(0, cx.poses)
        dk.set_draws(0, U)
        dk.step(steps)
        straight = dk.get_state(0)
    with sd.Docking([cx], tables, precision=sd.SD_PREC_FP64) as dk:
        dk.init_state(0, cx.poses)
        dk.set_draws(0, U[:, :stop, :])
        dk.step(stop)
        sd.write_checkpoint(tmp_path / "run.ckpt", dk.get_state(0), stop, steps)
    st, done, total = sd.read_checkpoint(tmp_path / "run.ckpt")
    assert done == stop and total == steps
    with sd.Docking([cx], tables, precision=sd.SD_PREC_FP64) as dk:
        dk.set_state(0, st)
        dk.set_draws(0, U[:, done:, :])
        dk.step(steps - done)
        resumed = dk.get_state(0)
    assert _equal(straight, resumed)


@pytest.mark.gpu
def test_mixed_state_restores_exactly(tmp_path, tables):
    cx = sd.SyntheticComplex(757, 481, 2, 64, seed=82)
    U = sd.gso_draws(6, cx.n_swarms, 6, cx.n_glowworms)
    with sd.Docking([cx], tables, precision=sd.SD_PREC_MIXED) as dk:
        dk.init_state(0, cx.poses)
        dk.set_draws(0, U[:, :3, :])
        dk.step(3)
        saved = dk.get_state(0)
        sd.write_checkpoint(tmp_path / "m.ckpt", saved, 3, 6)
    st, done, _ = sd.read_checkpoint(tmp_path / "m.ckpt")
    with sd.Docking([cx], tables, precision=sd.SD_PREC_MIXED) as dk:
        dk.set_state(0, st)
        assert _equal(dk.get_state(0), saved)
        dk.set_draws(0, U[:, done:, :])
        dk.step(3)
        assert (dk.get_state(0).step == saved.step + 3).all()
