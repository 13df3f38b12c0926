"""The drop-in, end to end: the reference's own entry point drives the library.

oracle/_ref/dropin_run is the reference's prepare_gso_tasks (source/dock/src/prepare_gso_tasks.cc,
compiled unmodified from its sources, with the configure-time path header its build generates)
called from a driver shaped like its main (reader, centring, normal-mode mask), with the hot-path
binding sparkledock_b200/bindings/cal_gso_tasks_b200.cc linked in place of its GPU translation
unit, over libsparkle_b200.so.  With USE_CUDA set, prepare_gso_tasks loads ./data/DCparams, types
the atoms with get_docking_model, computes the ligand reference point with its Eigen ellipsoid and
calls the binding, which runs the GSO steps on the GPU and writes swarm_<i>/gso_<steps>.out.
GPU test: in FP64 those files are byte-identical to the same files written from the oracle's
trajectory on the same inputs (the reference reader's coordinates and types, the reference's
ellipsoid point, the reference's draws); a mixed run ends with the same files' layout."""
import os
import subprocess

import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import OracleState, OracleSystem, _d, oracle_step, ref, ref_available, ref_structure

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin_run")
NM = 10


class ArraysComplex:
    """The fields of a complex the oracle reads, from plain arrays."""

    def __init__(self, rec_xyz, lig_xyz, rec_mask, lig_mask, rec_type, lig_type, rec_modes, lig_modes, lig_ref,
                 poses):
        self.rec_xyz, self.lig_xyz = rec_xyz, lig_xyz
        self.rec_mask, self.lig_mask = rec_mask.astype(np.int32), lig_mask.astype(np.int32)
        self.rec_type, self.lig_type = rec_type.astype(np.int32), lig_type.astype(np.int32)
        self.rec_modes, self.lig_modes = rec_modes, lig_modes
        self.n_rec, self.n_lig = len(rec_xyz), len(lig_xyz)
        self.n_modes_rec, self.n_modes_lig = rec_modes.shape[0], lig_modes.shape[0]
        self.n_swarms, self.n_glowworms = poses.shape[0], poses.shape[1]
        self.pose_len = poses.shape[2]
        self.poses = poses
        self.lig_ref = lig_ref
        self.rec_charge, self.lig_charge = np.zeros(self.n_rec), np.zeros(self.n_lig)
        self.rec_lj, self.lig_lj = np.zeros(self.n_rec, np.int32), np.zeros(self.n_lig, np.int32)


def dropin_inputs(folder, tables, S, G, seed=5):
    """Writes the run directory's inputs (PDB files, data/DCparams, poses and modes) and returns
    the driver's arguments."""
    rng = np.random.default_rng(seed)
    sd.synthetic_protein_pdb(str(folder / "rec.pdb"), 90, seed)
    sd.synthetic_protein_pdb(str(folder / "lig.pdb"), 40, seed + 1)
    (folder / "data").mkdir(exist_ok=True)
    with open(folder / "data" / "DCparams", "w") as f:
        f.write("".join("%.17g\n" % v for v in tables[0]))
    nr = sum(1 for ln in open(folder / "rec.pdb") if ln.startswith("ATOM"))
    nl = sum(1 for ln in open(folder / "lig.pdb") if ln.startswith("ATOM"))
    for name, n in (("rec_modes.bin", nr), ("lig_modes.bin", nl)):
        m = rng.normal(size=(NM, n, 3))
        m /= np.linalg.norm(m.reshape(NM, -1), axis=1)[:, None, None] / 0.5
        m.tofile(folder / name)
    pl = 7 + 2 * NM
    poses = np.zeros((S, G, pl))
    for s in range(S):
        d = rng.normal(size=3)
        c = d / np.linalg.norm(d) * 24.0
        for g in range(G):
            q = rng.normal(size=4)
            poses[s, g, :3] = c + rng.normal(scale=2.0, size=3)
            poses[s, g, 3:7] = q / np.linalg.norm(q)
            poses[s, g, 7:] = rng.normal(size=2 * NM)
    poses.tofile(folder / "poses.bin")
    return [str(folder / "rec.pdb"), str(folder / "lig.pdb"), str(folder / "poses.bin"), str(S), str(G), str(NM),
            str(NM), str(folder / "rec_modes.bin"), str(folder / "lig_modes.bin")]


def oracle_files(folder, tables, S, G, steps):
    """gso_<steps>.out text per swarm from the oracle's FP64 trajectory on the run's inputs."""
    from test_cli import gso_lines
    rx, rm, rt, _ = ref_structure(folder / "rec.pdb", False, False, False)
    lx, lm, lt, _ = ref_structure(folder / "lig.pdb", False, False, False)
    ref_pt = np.zeros(3)
    poles = np.zeros(18)
    ref().ref_min_volume_ellipsoid(_d(np.ascontiguousarray(lx)), len(lx), _d(ref_pt), _d(poles))
    pl = 7 + 2 * NM
    poses = np.fromfile(folder / "poses.bin").reshape(S, G, pl)
    cx = ArraysComplex(rx, lx, rm, lm, rt, lt, np.fromfile(folder / "rec_modes.bin").reshape(NM, len(rx), 3),
                       np.fromfile(folder / "lig_modes.bin").reshape(NM, len(lx), 3), ref_pt, poses)
    osys = OracleSystem(cx, tables)
    st = OracleState(S, G, pl, poses)
    U = sd.gso_draws(0, S, steps, G)
    for t in range(steps):
        oracle_step(osys, st, U[:, t, :])
    return gso_lines(st, pl)


@pytest.mark.gpu
def test_reference_entry_point_drives_the_library(tmp_path, tables):
    if not os.path.exists(DROPIN) or not ref_available():
        pytest.skip("oracle/_ref not built (the reference sources are needed to build it)")
    S, G, steps = 3, 40, 6
    args = dropin_inputs(tmp_path, tables, S, G)
    exp = oracle_files(tmp_path, tables, S, G, steps)
    for prec in ("fp64", "mixed"):
        run_dir = tmp_path / prec
        run_dir.mkdir()
        (run_dir / "data").symlink_to(tmp_path / "data")
        env = dict(os.environ, USE_CUDA="1", SPARKLE_STEPS=str(steps), SPARKLE_PRECISION=prec, NUM_THREADS="1")
        r = subprocess.run([DROPIN] + args, cwd=run_dir, capture_output=True, text=True, timeout=600, env=env)
        assert r.returncode == 0 and "sparkle_b200:" not in r.stderr, r.stderr[-3000:]
        assert "use cuda" in r.stdout and "dropin_run: done" in r.stdout
        for s in range(S):
            got = (run_dir / f"swarm_{s}" / f"gso_{steps}.out").read_text()
            if prec == "fp64":
                assert got == exp[s], f"swarm {s}: gso_{steps}.out differs from the oracle's"
            else:
                lines = got.splitlines()
                assert len(lines) == G + 1 and lines[0] == exp[s].splitlines()[0]
