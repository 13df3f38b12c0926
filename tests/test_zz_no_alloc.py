"""sd_score_poses_noalloc: the scoring entry point for callers that must not allocate device
memory while they score (graph capture, or a framework that owns all device memory).  It is
checked through the C ABI against the allocating entry point sd_score_poses on the same poses,
for two calls in a row (the second with other poses, so a stale scratch would show).
FP64: bit-identical; mixed: within 1e-5 relative, the mixed-precision tolerance of the other
GPU tests (the mixed kernel's summation order is dynamic, so two runs differ in the last bits).
This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import sparkledock_b200 as sd
from sparkledock_b200 import _abi

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry_point(tables):
    import torch
    cx = sd.SyntheticComplex(757, 481, 2, 60, seed=77)
    poses_all = np.ascontiguousarray(cx.poses.reshape(-1, cx.pose_len))
    with sd.Docking([cx], tables) as dk:
        for prec in (sd.SD_PREC_FP64, sd.SD_PREC_MIXED):
            for call, sl in enumerate((slice(0, 70), slice(50, 120))):
                poses = np.ascontiguousarray(poses_all[sl])
                n = poses.shape[0]
                ref_sc, ref_en = dk.score_poses(0, poses, prec)
                d_pose = torch.from_numpy(poses).cuda()
                d_sc = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
                d_en = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
                d_ref = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
                torch.cuda.synchronize()
                rc = _abi.lib().sd_score_poses_noalloc(dk._ctx, 0, C.c_void_p(d_pose.data_ptr()), n, prec,
                                                       C.c_void_p(d_sc.data_ptr()), C.c_void_p(d_en.data_ptr()),
                                                       C.c_void_p(d_ref.data_ptr()), 1)
                assert rc == 0, _abi.lib().sd_last_error()
                sc = d_sc.cpu().numpy()
                en = d_en.cpu().numpy()
                if prec == sd.SD_PREC_FP64:
                    assert np.array_equal(sc, ref_sc) and np.array_equal(en, ref_en), f"call {call}"
                else:
                    assert (np.abs(en - ref_en) / np.maximum(np.abs(ref_en), 1.0)).max() <= 1e-5, f"call {call}"
                assert np.isfinite(d_ref.cpu().numpy()).all()


def test_noalloc_rejects_oversized_calls(tables):
    cx = sd.SyntheticComplex(100, 80, 1, 4, seed=78)
    with sd.Docking([cx], tables) as dk:
        rc = _abi.lib().sd_score_poses_noalloc(dk._ctx, 0, C.c_void_p(16), 65537, sd.SD_PREC_MIXED,
                                               C.c_void_p(16), None, C.c_void_p(16), 1)
        assert rc == _abi.SD_ERR_ARG
        assert b"65536" in _abi.lib().sd_last_error()
