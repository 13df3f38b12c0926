"""Generates tests/golden/gso_small.npz from the reference's own compiled CPU functions
(oracle/_ref/libsdref.so, built from the reference tree by oracle/Makefile), on a complex
whose atoms use DFIRE types 0..11 only (the fixture stores that [12][12][20] table slice):
scores of the starting poses (cdfire_calculate_dfire + rotate + the reference's ANM loops)
and the state after 8 GSO steps driven over the reference's helpers with the reference's
draws (std::mt19937(0)).  The complex is a small seeded synthetic globule pair; all inputs are
stored in the fixture so that it is self-contained.

    python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

import sparkledock_b200 as sd  # noqa: E402
from oracle_bind import OracleState, OracleSystem, ref, ref_step  # noqa: E402


NT = 12


def expand_table(sub):
    t = np.zeros((168, 168, 20))
    t[:NT, :NT, :] = sub
    return t.ravel()


def main():
    cx = sd.SyntheticComplex(300, 200, 3, 40, 10, 10, seed=99)
    # 12 atom types keep the stored table slice small: types 0..11, table rows [12][12][20]
    cx.rec_type[:] %= NT
    cx.lig_type[:] %= NT
    full = sd.synthetic_tables(17)
    sub = full[0].reshape(168, 168, 20)[:NT, :NT, :].copy()
    tables = (expand_table(sub), full[1], full[2])
    osys = OracleSystem(cx, tables, cr_math=0)
    poses = np.ascontiguousarray(cx.poses.reshape(-1, cx.pose_len))
    dp = C.POINTER(C.c_double)
    scores0 = np.array([ref().ref_score_pose(osys.ptr, p.ctypes.data_as(dp), None, None, None) for p in poses])
    steps = 8
    U = np.empty((cx.n_swarms, steps, cx.n_glowworms))
    ref().ref_gso_draws(0, cx.n_swarms, steps, cx.n_glowworms, U.ctypes.data_as(dp))
    st = OracleState(cx.n_swarms, cx.n_glowworms, cx.pose_len, cx.poses)
    for t in range(steps):
        ref_step(osys, st, U[:, t, :], 1)
    np.savez_compressed(
        os.path.join(HERE, "gso_small.npz"),
        n_rec=cx.n_rec, n_lig=cx.n_lig, n_modes_rec=cx.n_modes_rec, n_modes_lig=cx.n_modes_lig,
        n_swarms=cx.n_swarms, n_glowworms=cx.n_glowworms,
        rec_xyz=cx.rec_xyz, lig_xyz=cx.lig_xyz, rec_mask=cx.rec_mask, lig_mask=cx.lig_mask,
        rec_modes=cx.rec_modes, lig_modes=cx.lig_modes, rec_type=cx.rec_type, lig_type=cx.lig_type,
        lig_ref=cx.lig_ref, table_sub=sub, poses=cx.poses, draws=U, scores0=scores0,
        final_pos=st.pos, final_luciferin=st.luciferin, final_vision=st.vision, final_select=st.select,
        final_nnei=st.nnei, final_scoring=st.scoring)
    print("moved after last step:", int(st.moved.sum()), "of", st.moved.size)


if __name__ == "__main__":
    main()
