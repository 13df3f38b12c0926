"""Swarm placement (sd_place_swarms) against the reference's calculate_start_pos.

CPU: the numpy restatement (oracle/place_oracle.py) against the reference's own
calculate_start_pos, compiled from its sources into oracle/_ref/libsdref_anm.so: swarm centres and
starting poses bit-identical.
GPU: sd_place_swarms against the same reference code: swarm centres and starting poses
bit-identical, for both surface-distance rules (ligand diameter below and above 20 A), with and
without ANM extents, and for a rank offset of the pose seed.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import sparkledock_b200 as sd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import place_oracle  # noqa: E402
from test_anm import ANM_SO, FLAGS, protein_pdb  # noqa: E402

_dp = C.POINTER(C.c_double)


def _ref_lib():
    if not os.path.exists(ANM_SO):
        pytest.skip("oracle/_ref/libsdref_anm.so not built (the reference sources are needed to build it)")
    L = C.CDLL(ANM_SO)
    L.ref_start_positions.restype = C.c_int
    L.ref_start_positions.argtypes = [C.c_char_p, C.c_char_p] + [C.c_int] * 10 + [C.c_double, _dp, _dp]
    return L


def ref_place(rec, lig, S, G, nmr, nml, use_anm, seed, anm_seed, radius=10.0):
    L = _ref_lib()
    cent = np.zeros((S, 3))
    poses = np.zeros((S, G, 7 + nmr + nml))
    n = L.ref_start_positions(str(rec).encode(), str(lig).encode(), 1, 1, 1, S, G, seed, anm_seed, nmr, nml,
                              int(use_anm), radius, cent.ctypes.data_as(_dp), poses.ctypes.data_as(_dp))
    assert n == S
    return cent, poses


# (receptor residues, ligand residues, swarms, glowworms, modes, seed); ligand of 5 residues:
# diameter below 20 A (surface distance 10 A); 40 or 60 residues: a quarter of its diameter
CASES = [(300, 60, 20, 8, 10, 11), (200, 5, 12, 5, 0, 12), (700, 40, 60, 4, 4, 13)]


@pytest.mark.parametrize("n_rec,n_lig,S,G,nm,seed", CASES)
def test_oracle_matches_reference_placement(tmp_path, n_rec, n_lig, S, G, nm, seed):
    protein_pdb(tmp_path / "rec.pdb", n_rec, seed)
    protein_pdb(tmp_path / "lig.pdb", n_lig, seed + 100)
    rc, rp = ref_place(tmp_path / "rec.pdb", tmp_path / "lig.pdb", S, G, nm, nm, nm > 0, seed, 7 * seed)
    rxyz, rnames, rfirst, rt = place_oracle.read_pdb(tmp_path / "rec.pdb")
    lxyz, _, _, _ = place_oracle.read_pdb(tmp_path / "lig.pdb")
    st = sd.Structure(tmp_path / "rec.pdb", FLAGS)
    assert np.array_equal(np.asarray(rt), st.translation)
    cent = place_oracle.swarm_centres(rxyz, rnames, rfirst, rt, lxyz, S)
    assert np.array_equal(cent, rc)
    poses = place_oracle.start_poses(cent, G, nm, nm, nm > 0, seed, 7 * seed)
    assert np.array_equal(poses, rp)


def test_oracle_library_draws():
    # std::mt19937 default-seeded (5489) is specified to give 4123659995 as its 10000th output
    g = place_oracle.MT19937(5489)
    for _ in range(9999):
        g()
    assert g() == 4123659995
    g = place_oracle.MT19937(1)
    vals = [place_oracle.uniform_int(g, 0, 6) for _ in range(2000)]
    assert min(vals) == 0 and max(vals) == 6
    assert all(0.0 <= place_oracle.uniform_double(g) < 1.0 for _ in range(1000))


@pytest.mark.gpu
@pytest.mark.parametrize("n_rec,n_lig,S,G,nm,seed", CASES + [(1500, 80, 150, 3, 10, 14)])
def test_place_swarms_matches_reference(tmp_path, n_rec, n_lig, S, G, nm, seed):
    protein_pdb(tmp_path / "rec.pdb", n_rec, seed)
    protein_pdb(tmp_path / "lig.pdb", n_lig, seed + 100)
    rc, rp = ref_place(tmp_path / "rec.pdb", tmp_path / "lig.pdb", S, G, nm, nm, nm > 0, seed, 7 * seed)
    rec, lig = sd.Structure(tmp_path / "rec.pdb", FLAGS), sd.Structure(tmp_path / "lig.pdb", FLAGS)
    cent, poses = sd.place_swarms(rec, lig, S, G, nm, nm, nm > 0, seed, 7 * seed)
    assert np.array_equal(cent, rc)
    assert np.array_equal(poses, rp)


@pytest.mark.gpu
def test_place_swarms_rank_and_radius(tmp_path):
    """The pose seed is starting_points_seed + rank (each MPI rank of the reference samples every
    swarm with its own seed); the swarm radius bounds each glowworm's offset."""
    protein_pdb(tmp_path / "rec.pdb", 250, 31)
    protein_pdb(tmp_path / "lig.pdb", 30, 32)
    rec, lig = sd.Structure(tmp_path / "rec.pdb", FLAGS), sd.Structure(tmp_path / "lig.pdb", FLAGS)
    c0, p0 = sd.place_swarms(rec, lig, 10, 20, 0, 0, False, 5, 6, swarm_radius=4.0)
    c1, p1 = sd.place_swarms(rec, lig, 10, 20, 0, 0, False, 4, 6, swarm_radius=4.0, rank=1)
    assert np.array_equal(c0, c1) and np.array_equal(p0, p1)
    off = np.linalg.norm(p0[:, :, :3] - c0[:, None, :], axis=2)
    assert off.max() <= 4.0 + 1e-12
    assert np.allclose(np.linalg.norm(p0[:, :, 3:7], axis=2), 1.0, atol=1e-12)


@pytest.mark.gpu
def test_place_swarms_errors(tmp_path):
    protein_pdb(tmp_path / "rec.pdb", 6, 41)
    protein_pdb(tmp_path / "lig.pdb", 4, 42)
    rec, lig = sd.Structure(tmp_path / "rec.pdb", FLAGS), sd.Structure(tmp_path / "lig.pdb", FLAGS)
    with pytest.raises(sd.SparkleError):
        sd.place_swarms(rec, lig, 40, 2)  # more swarms than surface atoms
    with pytest.raises(sd.SparkleError):
        sd.place_swarms(rec, lig, 0, 2)
    with pytest.raises(sd.SparkleError):
        sd.place_swarms(rec, lig, 2, 2, swarm_radius=0.0)
