"""lightdock_b200, the reference's command line (lightdock -f setup.json -s STEPS) over the C ABI.
CPU tests: argument and setup.json errors.  GPU test: the FP64 run's gso_<steps>.out files are
byte-identical to the same files written from the oracle's trajectory."""
import json
import os
import subprocess

import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import OracleState, OracleSystem, oracle_step

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
    assert r.returncode != 0 and "synthetic" in r.stderr
    sc = tmp_path / "sc.json"
    sc.write_text(json.dumps({"swarms": 2, "scoring": "vina", "synthetic": {"receptor_atoms": 50, "ligand_atoms": 40}}))
    r = run(["-f", str(sc)])
    assert r.returncode != 0 and "scoring" in r.stderr


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
