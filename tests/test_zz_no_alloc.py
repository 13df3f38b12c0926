"""sd_score_poses_noalloc: the scoring entry point for callers that must not allocate device
memory while they score (graph capture, or a framework that owns all device memory).  It is
checked through the C ABI against the allocating entry point sd_score_poses on the same poses,
for two calls in a row (the second with other poses, so a stale scratch would show), in every
precision and with both scoring functions: DFIRE scores and energies bit-identical (the mixed
kernel's summation order is fixed, so it too is reproducible to the bit); pyDock ones within
1e-10 (FP64) and 1e-5 (FP32) relative, since that kernel's per-lane sums follow the dynamic tile
order; ligand reference points bit-identical to the oracle's.  A non-finite pose is reported with sync; sync is refused while
the stream is being captured.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import OracleSystem, _d, oracle
from sparkledock_b200 import _abi

pytestmark = pytest.mark.gpu


def noalloc(dk, poses, prec, sync=1):
    import torch
    n = poses.shape[0]
    d_pose = torch.from_numpy(np.ascontiguousarray(poses)).cuda()
    d_sc = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    d_en = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    d_ref = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = _abi.lib().sd_score_poses_noalloc(dk._ctx, 0, C.c_void_p(d_pose.data_ptr()), n, prec,
                                           C.c_void_p(d_sc.data_ptr()), C.c_void_p(d_en.data_ptr()),
                                           C.c_void_p(d_ref.data_ptr()), sync)
    torch.cuda.synchronize()
    return rc, d_sc.cpu().numpy(), d_en.cpu().numpy(), d_ref.cpu().numpy()


def oracle_ref_points(cx, tables, poses):
    osys = OracleSystem(cx, tables)
    out = np.empty((len(poses), 3))
    lig = np.empty((cx.n_lig, 3))
    for k, p in enumerate(poses):
        oracle().or_ligand_pose(osys.ptr, _d(np.ascontiguousarray(p)), _d(lig), _d(out[k]))
    return out


@pytest.mark.parametrize("scoring", [sd.SD_SCORING_DFIRE, sd.SD_SCORING_PYDOCK], ids=["dfire", "pydock"])
def test_noalloc_matches_allocating_entry_point(scoring, tables):
    cx = sd.SyntheticComplex(757, 481, 2, 60, seed=77)
    poses_all = np.ascontiguousarray(cx.poses.reshape(-1, cx.pose_len))
    with sd.Docking([cx], tables, scoring=scoring) as dk:
        for prec in (sd.SD_PREC_FP64_REF, sd.SD_PREC_FP64, sd.SD_PREC_MIXED):
            for call, sl in enumerate((slice(0, 70), slice(50, 120))):
                poses = np.ascontiguousarray(poses_all[sl])
                ref_sc, ref_en = dk.score_poses(0, poses, prec)
                rc, sc, en, refp = noalloc(dk, poses, prec)
                assert rc == 0, _abi.lib().sd_last_error()
                if scoring == sd.SD_SCORING_DFIRE:
                    assert np.array_equal(sc, ref_sc) and np.array_equal(en, ref_en), f"precision {prec} call {call}"
                else:
                    tol = 1e-5 if prec == sd.SD_PREC_MIXED else 1e-10
                    err = np.abs(en - ref_en) / np.maximum(np.abs(ref_en), 1.0)
                    assert err.max() <= tol and np.array_equal(sc, -en), f"precision {prec} call {call}"
                assert np.array_equal(refp, oracle_ref_points(cx, tables, poses)), f"precision {prec} call {call}"


def test_noalloc_rejects_oversized_calls(tables):
    cx = sd.SyntheticComplex(100, 80, 1, 4, seed=78)
    with sd.Docking([cx], tables) as dk:
        rc = _abi.lib().sd_score_poses_noalloc(dk._ctx, 0, C.c_void_p(16), 65537, sd.SD_PREC_MIXED,
                                               C.c_void_p(16), None, C.c_void_p(16), 1)
        assert rc == _abi.SD_ERR_ARG
        assert b"65536" in _abi.lib().sd_last_error()


def test_noalloc_reports_non_finite_poses(tables):
    cx = sd.SyntheticComplex(300, 200, 1, 16, seed=79)
    poses = np.ascontiguousarray(cx.poses.reshape(-1, cx.pose_len)).copy()
    poses[3, 5] = np.nan
    poses[7, 0] = np.inf
    with sd.Docking([cx], tables) as dk:
        for prec in (sd.SD_PREC_FP64, sd.SD_PREC_MIXED):
            rc, _, _, _ = noalloc(dk, poses, prec, sync=1)
            assert rc == _abi.SD_ERR_NUMERIC
            assert b"2 non-finite" in _abi.lib().sd_last_error()
        rc, sc, _, _ = noalloc(dk, poses[:3], sd.SD_PREC_MIXED, sync=1)  # the finite ones still score
        assert rc == 0 and np.isfinite(sc).all()


def test_noalloc_refuses_sync_during_capture(tables):
    import torch
    cx = sd.SyntheticComplex(300, 200, 1, 16, seed=80)
    poses = np.ascontiguousarray(cx.poses.reshape(-1, cx.pose_len))
    with sd.Docking([cx], tables) as dk:
        rc, _, _, _ = noalloc(dk, poses, sd.SD_PREC_MIXED)  # first call on the device: before any capture
        assert rc == 0
        n = poses.shape[0]
        d_pose = torch.from_numpy(poses).cuda()
        d_sc = torch.empty(n, dtype=torch.float64, device="cuda")
        d_ref = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        stream = C.c_void_p()
        assert _abi.lib().sd_ctx_stream(dk._ctx, C.byref(stream)) == 0
        graph = torch.cuda.CUDAGraph()
        s = torch.cuda.ExternalStream(stream.value)
        with torch.cuda.stream(s):
            graph.capture_begin(capture_error_mode="relaxed")
            try:
                d_sc.zero_()  # something to capture, so that the graph is not empty
                rc = _abi.lib().sd_score_poses_noalloc(dk._ctx, 0, C.c_void_p(d_pose.data_ptr()), n, sd.SD_PREC_MIXED,
                                                       C.c_void_p(d_sc.data_ptr()), None,
                                                       C.c_void_p(d_ref.data_ptr()), 1)
            finally:
                graph.capture_end()
        torch.cuda.synchronize()
        assert rc == _abi.SD_ERR_ARG and b"capture" in _abi.lib().sd_last_error()
        del graph
