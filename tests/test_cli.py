"""lightdock_b200, the reference's command line (lightdock -f setup.json -s STEPS) over the C ABI.
CPU tests: argument and setup.json errors.  GPU test: the FP64 run's gso_<steps>.out files are
byte-identical to the same files written from the oracle's trajectory."""
import json
import os
import subprocess

import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import OracleState, OracleSystem, oracle_cluster, oracle_pose_atoms, oracle_step
from test_anm import protein_pdb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "sparkledock_b200", "lightdock_b200")


def run(args, cwd=None):
    return subprocess.run([CLI] + args, capture_output=True, text=True, cwd=cwd, timeout=300)


def test_cli_usage_and_setup_errors(tmp_path):
    r = run([])
    assert r.returncode != 0 and "usage" in r.stderr
    bad = tmp_path / "bad.json"
    bad.write_text('{"swarms": 2,, }')
    r = run(["-f", str(bad)])
    assert r.returncode != 0 and "setup.json" in r.stderr
    pdb = tmp_path / "pdb.json"
    pdb.write_text(json.dumps({"swarms": 2, "receptor_pdb": "r.pdb", "ligand_pdb": "l.pdb"}))
    r = run(["-f", str(pdb)])
    assert r.returncode != 0 and "cannot open" in r.stderr
    nopdb = tmp_path / "nopdb.json"
    nopdb.write_text(json.dumps({"swarms": 2}))
    r = run(["-f", str(nopdb)])
    assert r.returncode != 0 and "receptor_pdb" in r.stderr
    sc = tmp_path / "sc.json"
    sc.write_text(json.dumps({"swarms": 2, "scoring": "vina", "synthetic": {"receptor_atoms": 50, "ligand_atoms": 40}}))
    r = run(["-f", str(sc)])
    assert r.returncode != 0 and "scoring" in r.stderr
    # PDB inputs: option values checked before any device work
    protein_pdb(tmp_path / "r.pdb", 30, 1)
    protein_pdb(tmp_path / "l.pdb", 10, 2)
    for extra, word in (({"write_poses": "some"}, "write_poses"), ({"membrane": True}, "membrane"),
                        ({"dense_sampling": True}, "dense_sampling")):
        f = tmp_path / "opt.json"
        f.write_text(json.dumps({"swarms": 2, "receptor_pdb": "r.pdb", "ligand_pdb": "l.pdb", **extra}))
        r = run(["-f", str(f)], cwd=tmp_path)
        assert r.returncode != 0 and word in r.stderr, r.stderr


def gso_lines(st, pl):
    out = []
    for s in range(st.pos.shape[0]):
        lines = ["#Coordinates  RecID  LigID  Luciferin  Neighbor's number  Vision Range  Scoring"]
        for g in range(st.pos.shape[1]):
            lines.append("(" + ", ".join("%f" % v for v in st.pos[s, g]) + ")\t0\t0\t" + "%f" % st.luciferin[s, g] +
                         "\t" + str(st.nnei[s, g]) + "\t" + "%f" % st.vision[s, g] + "\t" + "%f" % st.scoring[s, g] +
                         "\t")
        out.append("\n".join(lines) + "\n")
    return out


@pytest.mark.gpu
def test_cli_fp64_run_matches_oracle(tmp_path, tables):
    setup = {"swarms": 2, "glowworms": 40, "anm_rec": 10, "anm_lig": 10, "use_anm": True, "precision": "fp64",
             "scoring": "dfire", "synthetic": {"receptor_atoms": 400, "ligand_atoms": 250, "seed": 12}}
    (tmp_path / "setup.json").write_text(json.dumps(setup))
    steps = 8
    r = run(["-f", "setup.json", "-s", str(steps)], cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert "simulation execution:" in r.stdout
    cx = sd.SyntheticComplex(400, 250, 2, 40, 10, 10, seed=12)
    osys = OracleSystem(cx, tables)
    st = OracleState(2, 40, cx.pose_len, cx.poses)
    U = sd.gso_draws(0, 2, steps, 40)
    for t in range(steps):
        oracle_step(osys, st, U[:, t, :])
    exp = gso_lines(st, cx.pose_len)
    for s in range(2):
        got = (tmp_path / f"swarm_{s}" / f"gso_{steps}.out").read_text()
        assert got == exp[s]
    info = json.loads((tmp_path / "run.json").read_text())
    assert (info["steps"], info["swarms"], info["glowworms"], info["precision"]) == (steps, 2, 40, "fp64")
    assert info["scored_poses"] >= 80 and info["seconds"]["gso"] > 0 and info["mixed_variant"] == -1


@pytest.mark.gpu
def test_cli_checkpoint_and_resume(tmp_path):
    """checkpoint_every writes checkpoint.ckpt without changing the run; a run stopped with -t and
    resumed with -r writes the same gso_<steps>.out files as the straight run; a checkpoint of a
    run with another -s is refused (the draws differ)."""
    setup = {"swarms": 2, "glowworms": 40, "anm_rec": 10, "anm_lig": 10, "use_anm": True, "precision": "fp64",
             "scoring": "dfire", "synthetic": {"receptor_atoms": 400, "ligand_atoms": 250, "seed": 13}}
    (tmp_path / "setup.json").write_text(json.dumps(setup))
    (tmp_path / "ck.json").write_text(json.dumps({**setup, "checkpoint_every": 2}))
    r = run(["-f", "setup.json", "-s", "6", "-o", "straight"], cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    r = run(["-f", "ck.json", "-s", "6", "-o", "chunked"], cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    r = run(["-f", "setup.json", "-s", "6", "-t", "4", "-o", "seg"], cwd=tmp_path)
    assert r.returncode == 0 and "stopped after step 4 of 6" in r.stdout, r.stderr
    assert not (tmp_path / "seg" / "swarm_0" / "gso_6.out").exists()
    _, done, total = sd.read_checkpoint(tmp_path / "seg" / "checkpoint.ckpt")
    assert (done, total) == (4, 6)
    r = run(["-f", "setup.json", "-s", "6", "-o", "seg", "-r", "seg/checkpoint.ckpt"], cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    for sw in range(2):
        ref = (tmp_path / "straight" / f"swarm_{sw}" / "gso_6.out").read_text()
        assert (tmp_path / "chunked" / f"swarm_{sw}" / "gso_6.out").read_text() == ref
        assert (tmp_path / "seg" / f"swarm_{sw}" / "gso_6.out").read_text() == ref
    r = run(["-f", "setup.json", "-s", "8", "-o", "other", "-r", "chunked/checkpoint.ckpt"], cwd=tmp_path)
    assert r.returncode != 0 and "6-step run" in r.stderr


@pytest.mark.gpu
def test_cli_pdb_inputs_match_oracle(tmp_path, tables):
    """PDB inputs through the command line: structures read as the reference's setup reads them,
    swarms placed by sd_place_swarms, ANM modes from sd_anm (which re-centres each structure),
    reference point from the final coordinates; the FP64 run's output files equal the oracle's
    trajectory on the same complex."""
    protein_pdb(tmp_path / "rec.pdb", 110, 31)
    protein_pdb(tmp_path / "lig.pdb", 45, 32)
    seed, S, G, steps = 19, 2, 40, 6
    setup = {"swarms": S, "glowworms": G, "anm_rec": 10, "anm_lig": 10, "use_anm": True, "precision": "fp64",
             "scoring": "dfire", "receptor_pdb": "rec.pdb", "ligand_pdb": "lig.pdb", "noxt": True, "noh": True,
             "now": True, "starting_points_seed": seed}
    (tmp_path / "setup.json").write_text(json.dumps(setup))
    r = run(["-f", "setup.json", "-s", str(steps)], cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    # the same complex built through the Python view of the ABI
    rs = sd.Structure(str(tmp_path / "rec.pdb"), sd.SD_PDB_NOXT | sd.SD_PDB_NOH | sd.SD_PDB_NOW)
    ls = sd.Structure(str(tmp_path / "lig.pdb"), sd.SD_PDB_NOXT | sd.SD_PDB_NOH | sd.SD_PDB_NOW)
    cx = sd.SyntheticComplex(rs.n_atoms, ls.n_atoms, S, G, 10, 10, seed=seed)
    cx.rec_xyz[:] = rs.xyz
    cx.rec_mask[:] = rs.nm_mask
    cx.rec_type[:] = rs.dfire_type
    cx.lig_xyz[:] = ls.xyz
    cx.lig_mask[:] = ls.nm_mask
    cx.lig_type[:] = ls.dfire_type
    _, poses = sd.place_swarms(rs, ls, S, G, 10, 10, True, seed, 324324)
    cx.rec_modes[:], cx.rec_xyz[:], _ = rs.anm(10, 0.5, S, G)
    cx.lig_modes[:], cx.lig_xyz[:], _ = ls.anm(10, 0.5, S, G)
    cx.lig_ref = sd.reference_point(cx.lig_xyz)
    osys = OracleSystem(cx, tables)
    st = OracleState(S, G, cx.pose_len, poses)
    U = sd.gso_draws(0, S, steps, G)
    for t in range(steps):
        oracle_step(osys, st, U[:, t, :])
    exp = gso_lines(st, cx.pose_len)
    for sw in range(S):
        got = (tmp_path / f"swarm_{sw}" / f"gso_{steps}.out").read_text()
        assert got == exp[sw]
    # cluster.repr from the oracle's clustering of the same final state on the CA atoms
    cl = oracle_cluster(osys, st.pos, st.scoring, rs.backbone, ls.backbone)
    for sw in range(S):
        lines = [f"{c}:{cl['size'][sw, c]}:{fmt_g(st.scoring[sw, cl['rep'][sw, c]])}:{cl['rep'][sw, c]}:"
                 f"lightdock_{cl['rep'][sw, c]}.pdb" for c in range(cl["n_clusters"][sw])]
        assert (tmp_path / f"swarm_{sw}" / "cluster.repr").read_text() == "\n".join(lines) + "\n"
    # one lightdock_<g>.pdb per representative, the oracle's final atoms in the reference's format
    for sw in range(S):
        reps = {int(cl["rep"][sw, c]) for c in range(cl["n_clusters"][sw])}
        files = {int(f.name[len("lightdock_"):-4]) for f in (tmp_path / f"swarm_{sw}").glob("lightdock_*.pdb")}
        assert files == reps
        for g in reps:
            r, l = oracle_pose_atoms(osys, st.pos[sw, g])
            sd.write_pose_pdb(tmp_path / "expected.pdb", rs, r, ls, l)
            assert (tmp_path / f"swarm_{sw}" / f"lightdock_{g}.pdb").read_bytes() == \
                (tmp_path / "expected.pdb").read_bytes()


def fmt_g(v):
    """A double as an ostream prints it by default (6 significant digits, %g)."""
    return "%g" % v
