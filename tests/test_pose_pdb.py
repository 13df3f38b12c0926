"""Pose files (sd_write_pose_pdb) against the reference's write_pdb.

CPU: the text written for given coordinates equals, byte for byte, what the reference's own
write_pdb (compiled from its sources into oracle/_ref/libsdref.so) writes for the same
structures and coordinates: synthetic chains with coordinates across the column range, records
with missing or malformed occupancy and B-factor fields, and the benchmark structures shipped with
the reference.  Coordinates that do not fit the columns are refused.
GPU: sd_materialise_poses gives the oracle's exact FP64 pose coordinates for chosen glowworms.
"""
import glob
import os

import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import OracleSystem, oracle_pose_atoms, ref, ref_available
from oracle_bind import _d as dp_

FLAGS = sd.SD_PDB_NOXT | sd.SD_PDB_NOH | sd.SD_PDB_NOW
REFERENCE = "/root/reference"


def _ref_text(rec_path, lig_path, rx, lx, out):
    if not ref_available():
        pytest.skip("oracle/_ref/libsdref.so not built")
    rx, lx = np.ascontiguousarray(rx), np.ascontiguousarray(lx)
    assert ref().ref_write_pose_pdb(str(rec_path).encode(), str(lig_path).encode(), 1, 1, 1, dp_(rx), dp_(lx),
                                    str(out).encode()) == 0
    return open(out).read()


def _coords(n, rng, lo=-999.0, hi=9999.0):
    x = rng.uniform(lo, hi, (n, 3))
    x[::7] = rng.uniform(-1.0, 1.0, (len(x[::7]), 3)) * 1e-3  # around zero, "-0.000" included
    return x


@pytest.mark.parametrize("seed", [1, 2])
def test_pose_file_matches_reference_writer(tmp_path, seed):
    rng = np.random.default_rng(seed)
    sd.synthetic_protein_pdb(tmp_path / "r.pdb", 120, seed)
    sd.synthetic_protein_pdb(tmp_path / "l.pdb", 40, seed + 10)
    r, l = sd.Structure(tmp_path / "r.pdb", FLAGS), sd.Structure(tmp_path / "l.pdb", FLAGS)
    rx, lx = _coords(r.n_atoms, rng), _coords(l.n_atoms, rng)
    sd.write_pose_pdb(tmp_path / "ours.pdb", r, rx, l, lx)
    assert open(tmp_path / "ours.pdb").read() == _ref_text(tmp_path / "r.pdb", tmp_path / "l.pdb", rx, lx,
                                                           tmp_path / "ref.pdb")


def test_pose_file_record_fields(tmp_path):
    """Alternate locations, insertion codes, chains, HETATM records, and occupancy / B-factor
    fields that are absent, short, unparsable or not consumed to their end."""
    lines = [
        "ATOM      1  N   GLY A   1      11.104   6.134  -6.504  1.00  0.00           N",
        "ATOM      2  CA AGLY A   1      11.639   6.071  -5.147  0.50 12.34           C",
        "ATOM      3  C   GLY A   1      12.000   7.000  -4.000",
        "ATOM      4  O   GLY A   1A     12.500   8.000  -4.500  1.0x  3.5",
        "HETATM    5  N   GLY B   2      10.000   5.000  -3.000  0.25 99.99",
        "ATOM      6  CA  GLY B   2       9.000   4.000  -2.000 1.00 2.00",
        "ATOM      7  C   GLY B   2       8.000   3.000  -1.000  1.00  0.0a",
        "ATOM      8  O   GLY    2       7.000   2.000   0.000  1.00-12.50",
    ]
    (tmp_path / "r.pdb").write_text("\n".join(lines) + "\nEND\n")
    sd.synthetic_protein_pdb(tmp_path / "l.pdb", 3, 4)
    r, l = sd.Structure(tmp_path / "r.pdb", FLAGS), sd.Structure(tmp_path / "l.pdb", FLAGS)
    rng = np.random.default_rng(5)
    rx, lx = _coords(r.n_atoms, rng, -50, 50), _coords(l.n_atoms, rng, -50, 50)
    sd.write_pose_pdb(tmp_path / "ours.pdb", r, rx, l, lx)
    assert open(tmp_path / "ours.pdb").read() == _ref_text(tmp_path / "r.pdb", tmp_path / "l.pdb", rx, lx,
                                                           tmp_path / "ref.pdb")


def test_pose_file_benchmark_structures(tmp_path):
    files = sorted(glob.glob(os.path.join(REFERENCE, "**", "*_r_u.pdb"), recursive=True))
    if not files:
        pytest.skip("reference tree not present")
    rng = np.random.default_rng(9)
    for rp in files[:4]:
        lp = rp.replace("_r_u.pdb", "_l_u.pdb")
        r, l = sd.Structure(rp, FLAGS), sd.Structure(lp, FLAGS)
        rx, lx = r.xyz + rng.normal(0, 20, 3), l.xyz + rng.normal(0, 20, 3)
        sd.write_pose_pdb(tmp_path / "ours.pdb", r, rx, l, lx)
        assert open(tmp_path / "ours.pdb").read() == _ref_text(rp, lp, rx, lx, tmp_path / "ref.pdb"), rp


def test_pose_file_refuses_wide_fields(tmp_path):
    sd.synthetic_protein_pdb(tmp_path / "r.pdb", 5, 1)
    r = sd.Structure(tmp_path / "r.pdb", FLAGS)
    x = np.zeros((r.n_atoms, 3))
    x[3, 1] = 10000.0  # "10000.000": nine columns
    with pytest.raises(sd.SparkleError):
        sd.write_pose_pdb(tmp_path / "o.pdb", r, x)
    x[3, 1] = -1000.0
    with pytest.raises(sd.SparkleError):
        sd.write_pose_pdb(tmp_path / "o.pdb", r, x)
    x[3, 1] = 9999.9994  # rounds to 9999.999: fits
    sd.write_pose_pdb(tmp_path / "o.pdb", r, x)
    assert "9999.999" in open(tmp_path / "o.pdb").read()


@pytest.mark.gpu
def test_materialise_matches_oracle(tables):
    """Final all-atom coordinates of chosen glowworms after a few FP64 GSO steps, bit-identical to
    the oracle's transforms of the same final poses; a batch larger than one launch's chunk is
    not needed for this (the chunking only splits the pose list)."""
    cx = sd.SyntheticComplex(600, 300, 3, 20, 10, 10, seed=5)
    idx = np.array([0, 5, 21, 59, 33, 40])
    with sd.Docking([cx], tables, precision=sd.SD_PREC_FP64) as dk:
        dk.init_state(0, cx.poses)
        dk.set_draws(0, sd.gso_draws(0, 3, 4, 20))
        dk.step(4)
        st = dk.get_state(0)
        rec, lig = dk.materialise(0, idx)
        with pytest.raises(sd.SparkleError):
            dk.materialise(0, [60])
    osys = OracleSystem(cx, tables)
    flat = st.pos.reshape(-1, cx.pose_len)
    for k, i in enumerate(idx):
        r, l = oracle_pose_atoms(osys, flat[i])
        assert np.array_equal(rec[k], r) and np.array_equal(lig[k], l), i
