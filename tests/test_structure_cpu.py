"""Structures from PDB files: the C-ABI loader against the reference's own setup code
(read_input_structure + init_center_translate + translate + get_nm_mask + get_docking_model,
compiled from its sources) on the benchmark structures shipped with the reference, and the
parsing rules on small hand-written files."""
import glob
import os

import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import ref_available, ref_structure

REF_BM = "/root/reference/bm"
PDBS = sorted(glob.glob(os.path.join(REF_BM, "*", "*_u.pdb")))
needs_ref = pytest.mark.skipif(not (ref_available() and PDBS), reason="reference tree or harness not available")


@needs_ref
@pytest.mark.parametrize("flags", [(True, True, True), (False, False, False)])
def test_structures_match_reference_setup(flags):
    noxt, noh, now = flags
    f = (sd.SD_PDB_NOXT if noxt else 0) | (sd.SD_PDB_NOH if noh else 0) | (sd.SD_PDB_NOW if now else 0)
    for path in PDBS:
        xyz, mask, dfire, tr = ref_structure(path, noxt, noh, now)
        try:
            s = sd.Structure(path, f)
        except sd.SparkleError as e:
            # without the noxt filter an OXT atom has no DFIRE type: the reference reads an
            # uninitialised table index there, the loader reports it
            assert not noxt and "DFIRE" in str(e), (path, e)
            continue
        assert s.n_atoms == len(xyz), path
        assert np.array_equal(s.xyz, xyz), path
        assert np.array_equal(s.translation, tr), path
        assert np.array_equal(s.nm_mask, mask), path
        assert np.array_equal(s.dfire_type, dfire), path


@needs_ref
def test_benchmark_structure_sizes():
    """With the reference's default filters the ten complexes have the atom counts the
    benchmark configurations use (e.g. 3002 / 1274 for the single-complex workload)."""
    counts = {os.path.basename(p): sd.Structure(p, sd.SD_PDB_NOXT | sd.SD_PDB_NOH | sd.SD_PDB_NOW).n_atoms
              for p in PDBS}
    assert counts.get("2VXT_r_u.pdb") == 3002 and counts.get("2VXT_l_u.pdb") == 1274
    assert counts.get("4GAM_r_u.pdb") == 17307 and counts.get("4GAM_l_u.pdb") == 1125


def _atom(serial, name, res, chain, resnum, x, y, z, ins=" ", rec="ATOM"):
    nm = (" " + name) if len(name) < 4 else name
    return f"{rec:<6}{serial:5d} {nm:<4} {res:<3} {chain}{resnum:4d}{ins}   {x:8.3f}{y:8.3f}{z:8.3f}  1.00  0.00\n"


def test_parsing_rules(tmp_path):
    """First MODEL only, noh/noxt/now filters, residues split on insertion codes, coordinates
    through float, centre = mean of the non-hydrogen atoms, mask and DFIRE types."""
    lines = ["MODEL        1\n",
             _atom(1, "N", "GLY", "A", 1, 1.111, 2.222, 3.333),
             _atom(2, "CA", "GLY", "A", 1, 2.5, 2.0, 3.0),
             _atom(3, "H", "GLY", "A", 1, 9.0, 9.0, 9.0),
             _atom(4, "C", "GLY", "A", 1, 3.0, 2.5, 3.5),
             _atom(5, "O", "GLY", "A", 1, 3.5, 3.5, 3.5),
             _atom(6, "N", "GLY", "A", 1, 4.0, 4.0, 4.0, ins="A"),
             _atom(7, "CA", "GLY", "A", 1, 5.0, 4.0, 4.0, ins="A"),
             _atom(8, "OXT", "GLY", "A", 1, 6.0, 4.0, 4.0, ins="A"),
             _atom(9, "O", "HOH", "W", 2, 7.0, 7.0, 7.0, rec="HETATM"),
             "ENDMDL\n", "MODEL        2\n",
             _atom(1, "N", "ALA", "A", 1, 50.0, 50.0, 50.0),
             "ENDMDL\n"]
    p = tmp_path / "t.pdb"
    p.write_text("".join(lines))
    s = sd.Structure(str(p), sd.SD_PDB_NOXT | sd.SD_PDB_NOH | sd.SD_PDB_NOW)
    assert s.n_atoms == 6 and s.n_residues == 2  # GLY 1 and GLY 1A; the second MODEL is ignored
    raw = np.array([[1.111, 2.222, 3.333], [2.5, 2, 3], [3, 2.5, 3.5], [3.5, 3.5, 3.5], [4, 4, 4],
                    [5, 4, 4]]).astype(np.float32).astype(np.float64)
    centre = -1 * raw.sum(0) / 6
    assert np.array_equal(s.translation, centre)
    assert np.array_equal(s.xyz, raw + centre)
    assert list(s.nm_mask) == [1] * 6
    assert list(s.backbone) == [0, 1, 0, 0, 0, 1]
    assert list(s.dfire_type) == [79, 80, 81, 82, 79, 80]
    # without a filter the water, the hydrogen or the OXT atom has no DFIRE type
    for flags in (sd.SD_PDB_NOXT | sd.SD_PDB_NOH, sd.SD_PDB_NOXT | sd.SD_PDB_NOW, sd.SD_PDB_NOH | sd.SD_PDB_NOW):
        with pytest.raises(sd.SparkleError) as e:
            sd.Structure(str(p), flags)
        assert "DFIRE" in str(e.value)


def test_loader_errors(tmp_path):
    p = tmp_path / "bad.pdb"
    p.write_text(_atom(1, "XX", "GLY", "A", 1, 0, 0, 0))
    with pytest.raises(sd.SparkleError) as e:
        sd.Structure(str(p))
    assert "element" in str(e.value)
    p.write_text(_atom(1, "CZ", "GLY", "A", 1, 0, 0, 0))
    with pytest.raises(sd.SparkleError) as e:
        sd.Structure(str(p))
    assert "DFIRE" in str(e.value)
    with pytest.raises(sd.SparkleError):
        sd.Structure(str(tmp_path / "missing.pdb"))
    p.write_text("REMARK nothing\n")
    with pytest.raises(sd.SparkleError):
        sd.Structure(str(p))


def test_starting_poses_match_synthetic_generator():
    """sd_starting_poses on a receptor reproduces the synthetic generator's poses for the same
    seed (one routine behind both)."""
    cx = sd.SyntheticComplex(300, 200, 3, 16, 10, 10, seed=77)
    poses = np.empty_like(cx.poses)
    assert sd._abi.lib().sd_starting_poses(sd.dptr(cx.rec_xyz), 300, 3, 16, 10, 10, 77, sd.dptr(poses)) == 0
    assert np.array_equal(poses, cx.poses)
    ref = np.empty(3)
    assert sd._abi.lib().sd_reference_point(sd.dptr(cx.lig_xyz), 200, sd.dptr(ref)) == 0
    assert np.array_equal(ref, cx.lig_ref)


@needs_ref
def test_reference_point_matches_reference_ellipsoid():
    """sd_reference_point (Khachiyan MVEE centre, tolerance 0.01, restated in the operation order of
    the reference's minimum_volume_ellipsoid and of the Eigen inverse it calls) is bit-identical to
    the reference's own compiled function on random point clouds of many shapes and sizes and on every
    ligand of the benchmark structures shipped with the reference; so is the oracle's independent
    restatement.  The reference runs single-threaded here (NUM_THREADS unset): with more threads
    its weight-change sum is a data race."""
    import ctypes as C
    from oracle_bind import oracle, ref
    dp = C.POINTER(C.c_double)
    rng = np.random.default_rng(0)
    clouds = [np.ascontiguousarray(rng.normal(size=(int(rng.integers(4, 1500)), 3)) * rng.uniform(0.5, 30, 3) +
                                   rng.uniform(-50, 50, 3)) for _ in range(30)]
    clouds += [sd.Structure(p, sd.SD_PDB_NOXT | sd.SD_PDB_NOH | sd.SD_PDB_NOW).xyz for p in PDBS if "_l_" in p]
    assert len(clouds) == 40
    for pts in clouds:
        pts = np.ascontiguousarray(pts)
        a, c, o, poles = np.empty(3), np.empty(3), np.empty(3), np.empty(18)
        assert sd._abi.lib().sd_reference_point(sd.dptr(pts), len(pts), sd.dptr(a)) == 0
        ref().ref_min_volume_ellipsoid(pts.ctypes.data_as(dp), len(pts), c.ctypes.data_as(dp), poles.ctypes.data_as(dp))
        oracle().or_mvee_center(pts.ctypes.data_as(dp), len(pts), 0.01, o.ctypes.data_as(dp))
        assert np.array_equal(a, c), (len(pts), a - c)
        assert np.array_equal(o, c), (len(pts), o - c)
