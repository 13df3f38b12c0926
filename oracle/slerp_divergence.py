"""Test infrastructure (a measurement, not part of the product): how far a GSO trajectory with the
correctly rounded acos and sin that this build's slerp uses drifts from the reference's own
trajectory, which calls the platform libm.

Trajectory A: the reference's own compiled GSO helpers and scorer (prepare_gso_tasks.cc, built
unmodified into oracle/_ref/libsdref.so), driven step by step (tests/oracle_bind.py ref_step).
Trajectory B: the oracle with cr_math = 1, whose every step is bit-identical to the GPU's (the GPU
parity tests pin that).  Both start from the same poses and use the same draws (std::mt19937(0)).
Reported per step: the fraction of glowworms whose state differs in any field (position,
luciferin, vision range, neighbour count, selection, score, reference point), the fraction whose
position differs, and the largest position difference.

Inputs: the first benchmark configuration's synthetic complex (757 / 481 atoms, 130 swarms x 200
glowworms, seed 100, the benchmark's own generator restated by the oracle) and the benchmark
structures shipped with the reference (its bm/ directory: coordinates, masks and DFIRE types from
the reference's own reader, starting poses from its own calculate_start_pos, seeded random
orthonormal normal modes), a few swarms each so that the CPU finishes in minutes.

    python oracle/slerp_divergence.py [--steps 100] [--bm-swarms 2] [--out FILE]
"""
import argparse
import ctypes as C
import glob
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from oracle_bind import (OracleState, OracleSynthComplex, OracleSystem, oracle_draws, oracle_step,  # noqa: E402
                         oracle_tables, ref, ref_step, ref_structure)

REF_BM = "/root/reference/bm"
FIELDS = (("pos", 27), ("scoring", 1), ("luciferin", 1), ("vision", 1), ("nnei", 1), ("select", 1), ("ref", 3))


class BmComplex:
    """A benchmark structure pair set up by the reference's own code (reader, centring, mask, DFIRE
    types, calculate_start_pos), with seeded random orthonormal normal modes."""

    def __init__(self, rec_pdb, lig_pdb, n_swarms, n_glowworms, seed):
        rx, rm, rt, _ = ref_structure(rec_pdb, True, True, True)
        lx, lm, lt, _ = ref_structure(lig_pdb, True, True, True)
        self.rec_xyz, self.lig_xyz = rx, lx
        self.rec_mask, self.lig_mask = rm.astype(np.int32), lm.astype(np.int32)
        self.rec_type, self.lig_type = rt.astype(np.int32), lt.astype(np.int32)
        self.n_rec, self.n_lig = len(rx), len(lx)
        self.n_modes_rec = self.n_modes_lig = 10
        rng = np.random.default_rng(seed)
        self.rec_modes = self._modes(rng, self.n_rec)
        self.lig_modes = self._modes(rng, self.n_lig)
        self.n_glowworms = n_glowworms
        self.pose_len = 27
        placed = 50
        L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libsdref_anm.so"))
        dp = C.POINTER(C.c_double)
        L.ref_start_positions.argtypes = [C.c_char_p, C.c_char_p] + [C.c_int] * 10 + [C.c_double, dp, dp]
        cent = np.zeros((placed, 3))
        poses = np.zeros((placed, n_glowworms, 27))
        sys.stdout.flush()
        saved = os.dup(1)
        os.dup2(2, 1)  # the reference reports its progress on stdout
        try:
            rc = L.ref_start_positions(rec_pdb.encode(), lig_pdb.encode(), 1, 1, 1, placed, n_glowworms, 324324,
                                       324324, 10, 10, 1, 10.0, cent.ctypes.data_as(dp), poses.ctypes.data_as(dp))
        finally:
            os.dup2(saved, 1)
            os.close(saved)
        assert rc == placed  # the number of swarms placed
        self.n_swarms = n_swarms
        self.poses = np.ascontiguousarray(poses[:n_swarms])
        c = np.zeros(3)
        poles = np.zeros(18)
        ref().ref_min_volume_ellipsoid(np.ascontiguousarray(lx).ctypes.data_as(dp), self.n_lig, c.ctypes.data_as(dp),
                                       poles.ctypes.data_as(dp))
        self.lig_ref = c
        self.rec_charge, self.lig_charge = np.zeros(self.n_rec), np.zeros(self.n_lig)
        self.rec_lj, self.lig_lj = np.zeros(self.n_rec, np.int32), np.zeros(self.n_lig, np.int32)

    @staticmethod
    def _modes(rng, n):
        m = rng.normal(size=(10, n, 3))
        m /= np.linalg.norm(m.reshape(10, -1), axis=1)[:, None, None]
        return np.ascontiguousarray(m * np.sqrt(n) * 0.1)


def diverge(cx, tables, steps, threads):
    osys_ref = OracleSystem(cx, tables, cr_math=0)
    osys_cr = OracleSystem(cx, tables, cr_math=1)
    a = OracleState(cx.n_swarms, cx.n_glowworms, cx.pose_len, cx.poses)
    b = OracleState(cx.n_swarms, cx.n_glowworms, cx.pose_len, cx.poses)
    U = oracle_draws(0, cx.n_swarms, steps, cx.n_glowworms)
    n = cx.n_swarms * cx.n_glowworms
    any_frac, pos_frac, pos_max = [], [], []
    for t in range(steps):
        ref_step(osys_ref, a, U[:, t, :], threads)
        oracle_step(osys_cr, b, U[:, t, :], nthreads=threads)
        diff = np.zeros(n, bool)
        for f, w in FIELDS:
            x = getattr(a, f).reshape(n, w)
            y = getattr(b, f).reshape(n, w)
            diff |= (x != y).any(axis=1)
        dp = np.abs(a.pos - b.pos).reshape(n, -1)
        any_frac.append(float(diff.mean()))
        pos_frac.append(float((dp > 0).any(axis=1).mean()))
        pos_max.append(float(dp.max()))
    first = next((t for t, f in enumerate(any_frac) if f > 0), None)
    return {"swarms": cx.n_swarms, "glowworms": cx.n_glowworms, "receptor_atoms": cx.n_rec,
            "ligand_atoms": cx.n_lig, "steps": steps, "first_step_with_a_difference": first,
            "fraction_differing_any_field": any_frac, "fraction_differing_position": pos_frac,
            "max_position_difference": pos_max}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--bm-swarms", type=int, default=2)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default="")
    args = ap.parse_args()
    tables = oracle_tables(3)
    res = {"steps": args.steps, "threads": args.threads, "complexes": {}}
    t0 = time.time()
    cx = OracleSynthComplex(757, 481, 130, 200, 10, 10, seed=100)
    res["complexes"]["synthetic 757/481, 130 x 200"] = diverge(cx, tables, args.steps, args.threads)
    print("synthetic done", time.time() - t0, file=sys.stderr)
    for rec in sorted(glob.glob(os.path.join(REF_BM, "*", "*_r_u.pdb"))):
        lig = rec.replace("_r_u.pdb", "_l_u.pdb")
        name = os.path.basename(os.path.dirname(rec))
        cx = BmComplex(rec, lig, args.bm_swarms, 200, seed=7)
        res["complexes"][name] = diverge(cx, tables, args.steps, args.threads)
        print(name, time.time() - t0, file=sys.stderr)
    text = json.dumps(res)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)
    print(text)


if __name__ == "__main__":
    main()
