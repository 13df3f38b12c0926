"""Seeded random PDB files through the loader and the pose writer, against the reference's own
reader and write_pdb (compiled from its sources): atom counts, coordinates, centring, mask and
DFIRE types equal, and the written pose files equal byte for byte.  The files vary the record
type, alternate locations, chains, insertion codes, residue numbering (gaps, negative numbers),
occupancy and B-factor fields (present, absent, malformed), interleaved TER / REMARK lines, CRLF
line endings and a second MODEL; every atom belongs to a residue with DFIRE types (GLY, ALA, SER),
where both readers are defined."""
import numpy as np
import pytest

import sparkledock_b200 as sd
from oracle_bind import _d as dp_
from oracle_bind import ref, ref_available, ref_structure

RESIDUES = {"GLY": ["N", "CA", "C", "O"], "ALA": ["N", "CA", "C", "O", "CB"],
            "SER": ["N", "CA", "C", "O", "CB", "OG"]}
FLAGS = sd.SD_PDB_NOXT | sd.SD_PDB_NOH | sd.SD_PDB_NOW
needs_ref = pytest.mark.skipif(not ref_available(), reason="reference harness not built")


def fuzz_pdb(path, seed, n_res=60):
    rng = np.random.default_rng(seed)
    lines, serial, resnum = [], 1, int(rng.integers(-20, 50))
    if rng.random() < 0.5:
        lines.append("MODEL        1")
    for r in range(n_res):
        res = ["GLY", "ALA", "SER"][int(rng.integers(0, 3))]
        resnum += int(rng.choice([1, 1, 1, 2, 5]))
        ins = " " if rng.random() < 0.85 else "ABC"[int(rng.integers(0, 3))]
        chain = "ABZ"[int(rng.integers(0, 3))] if rng.random() < 0.3 else "A"
        rec = "HETATM" if rng.random() < 0.1 else "ATOM  "
        for name in RESIDUES[res]:
            x, y, z = rng.normal(0, 15, 3)
            alt = " " if rng.random() < 0.9 else "A"
            nm = (" " + name) if len(name) < 4 else name
            tail = rng.random()
            if tail < 0.55:
                extra = f"{rng.uniform(0, 1):6.2f}{rng.uniform(0, 99):6.2f}          {name[0]:>2}"
            elif tail < 0.7:
                extra = ""  # no occupancy or B-factor
            elif tail < 0.8:
                extra = f"{rng.uniform(0, 1):6.2f}"  # occupancy only
            elif tail < 0.9:
                extra = "  1.0x 12.5"  # malformed occupancy
            else:
                extra = f" {rng.uniform(0, 1):5.2f}{rng.uniform(0, 9):5.2f}  "  # fields ending early
            lines.append(f"{rec}{serial:5d} {nm:<4}{alt}{res:<3} {chain}{resnum:4d}{ins}   "
                         f"{x:8.3f}{y:8.3f}{z:8.3f}{extra}")
            serial += 1
        if rng.random() < 0.05:
            lines.append("TER")
        if rng.random() < 0.05:
            lines.append("REMARK   a remark between residues")
    if lines[0].startswith("MODEL"):
        lines += ["ENDMDL", "MODEL        2", f"ATOM  {serial:5d}  N   GLY A 999       1.000   2.000   3.000",
                  "ENDMDL"]
    eol = "\r\n" if rng.random() < 0.3 else "\n"
    with open(path, "w", newline="") as f:
        f.write(eol.join(lines) + eol + "END" + eol)


@needs_ref
@pytest.mark.parametrize("seed", range(16))
def test_fuzz_files_match_reference_reader_and_writer(tmp_path, seed):
    p = tmp_path / "f.pdb"
    fuzz_pdb(p, seed)
    xyz, mask, dfire, tr = ref_structure(p, True, True, True)
    s = sd.Structure(p, FLAGS)
    assert s.n_atoms == len(xyz)
    assert np.array_equal(s.xyz, xyz) and np.array_equal(s.translation, tr)
    assert np.array_equal(s.nm_mask, mask) and np.array_equal(s.dfire_type, dfire)
    # the pose writer, receptor and ligand both this structure, moved apart
    rx = np.ascontiguousarray(s.xyz)
    lx = np.ascontiguousarray(s.xyz + np.array([40.0, -30.0, 5.0]))
    sd.write_pose_pdb(tmp_path / "ours.pdb", s, rx, s, lx)
    assert ref().ref_write_pose_pdb(str(p).encode(), str(p).encode(), 1, 1, 1, dp_(rx), dp_(lx),
                                    str(tmp_path / "ref.pdb").encode()) == 0
    assert (tmp_path / "ours.pdb").read_bytes() == (tmp_path / "ref.pdb").read_bytes()
