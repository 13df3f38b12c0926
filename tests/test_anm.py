"""ANM normal modes (sd_anm) against the reference's cal_anm.

CPU: the numpy restatement (oracle/anm_oracle.py) against the reference's own compiled functions:
the Hessian (build_hessian1D) and the re-centring (norm) bit-identical, and the extent draws
bit-identical to std::default_random_engine + std::normal_distribution.
GPU: sd_anm against the reference's cal_anm run unmodified with its cuSOLVER eigensolver
(oracle/_ref/libsdref_anm.so, in a child process), and against the numpy restatement (modes within
1e-8 of the largest component after aligning each mode's sign, eigenvalues within 1e-10 relative).
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

import sparkledock_b200 as sd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import anm_oracle  # noqa: E402

ANM_SO = os.path.join(ROOT, "oracle", "_ref", "libsdref_anm.so")
FLAGS = sd.SD_PDB_NOXT | sd.SD_PDB_NOH | sd.SD_PDB_NOW
_dp = C.POINTER(C.c_double)


protein_pdb = sd.synthetic_protein_pdb


def _anm_lib():
    if not os.path.exists(ANM_SO):
        pytest.skip("oracle/_ref/libsdref_anm.so not built (the reference sources are needed to build it)")
    L = C.CDLL(ANM_SO)
    L.ref_build_hessian.argtypes = [_dp, C.c_int, _dp]
    L.ref_norm.argtypes = [_dp, C.c_int]
    L.harness_extent_coef.restype = C.c_double
    L.harness_extent_coef.argtypes = [_dp, C.c_int, C.c_longlong]
    return L


def _p(a):
    return a.ctypes.data_as(_dp)


@pytest.mark.parametrize("n_res,seed", [(40, 1), (250, 2)])
def test_oracle_hessian_matches_reference(tmp_path, n_res, seed):
    L = _anm_lib()
    names, _ = protein_pdb(tmp_path / "p.pdb", n_res, seed)
    st = sd.Structure(tmp_path / "p.pdb", FLAGS)
    xyz = anm_oracle.recentre(st.xyz)
    ref = np.ascontiguousarray(st.xyz.copy())
    L.ref_norm(_p(ref), st.n_atoms)
    assert np.array_equal(xyz, ref)
    nodes = np.ascontiguousarray(anm_oracle.nodes_of(xyz, names))
    H = np.empty((3 * n_res, 3 * n_res))
    L.ref_build_hessian(_p(nodes), n_res, _p(H))
    H2 = anm_oracle.hessian(nodes)
    assert np.array_equal(H, H2)
    assert np.array_equal(H2, H2.T)
    # translations are zero modes: every row sums to zero (to rounding)
    assert np.abs(H2.reshape(3 * n_res, n_res, 3).sum(axis=1)).max() < 1e-12


@pytest.mark.parametrize("n_modes,n_draws", [(10, 2000), (1, 7), (20, 3)])
def test_oracle_extent_draws_match_cpp_library(n_modes, n_draws):
    L = _anm_lib()
    lam = np.random.default_rng(n_modes).uniform(0.01, 3.0, n_modes)
    assert anm_oracle.extent_coef(lam, n_draws) == L.harness_extent_coef(_p(lam), n_modes, n_draws)


def test_oracle_six_zero_modes(tmp_path):
    names, first = protein_pdb(tmp_path / "p.pdb", 60, 5)
    st = sd.Structure(tmp_path / "p.pdb", FLAGS)
    H = anm_oracle.hessian(anm_oracle.nodes_of(anm_oracle.recentre(st.xyz), names))
    w = np.linalg.eigvalsh(H)
    assert np.sum(w < anm_oracle.ZERO_EIGENVALUE) == 6 and w[6] > 1e-4
    modes, _, lam = anm_oracle.anm(st.xyz, names, first, 8, 0.5, 3, 10)
    assert modes.shape == (8, st.n_atoms, 3) and np.all(np.diff(lam) >= 0)
    # atoms of one residue move together; over the nodes (CA atoms) each mode is orthogonal to
    # rigid translations
    for r in range(len(first) - 1):
        assert np.array_equal(modes[:, first[r]], modes[:, first[r + 1] - 1])
    ca = [i for i, n in enumerate(names) if n == "CA"]
    assert np.abs(modes[:, ca].sum(axis=1)).max() < 1e-9 * np.abs(modes).max() * len(ca)


def _align_signs(a, b):
    s = np.sign(np.einsum("mij,mij->m", a, b))
    return b * s[:, None, None]


@pytest.mark.gpu
@pytest.mark.parametrize("n_res,n_modes,seed", [(120, 10, 11), (700, 10, 12), (300, 20, 13)])
def test_anm_matches_reference_cal_anm(tmp_path, n_res, n_modes, seed):
    if not os.path.exists(ANM_SO):
        pytest.skip("oracle/_ref/libsdref_anm.so not built")
    protein_pdb(tmp_path / "p.pdb", n_res, seed)
    rmsd, S, G = 0.5, 25, 40
    child = os.path.join(os.path.dirname(__file__), "ref_anm_child.py")
    r = subprocess.run([sys.executable, child, str(tmp_path / "p.pdb"), str(n_modes), str(rmsd), str(S), str(G),
                        str(tmp_path / "ref.npz")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    ref = np.load(tmp_path / "ref.npz")
    modes, xyz, lam = sd.Structure(tmp_path / "p.pdb", FLAGS).anm(n_modes, rmsd, S, G)
    assert np.array_equal(xyz, ref["xyz"])
    assert np.array_equal(modes, ref["modes"]), np.abs(modes - ref["modes"]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("n_res,n_modes,seed", [(150, 10, 21), (400, 12, 22)])
def test_anm_matches_numpy_oracle(tmp_path, n_res, n_modes, seed):
    names, first = protein_pdb(tmp_path / "p.pdb", n_res, seed)
    st = sd.Structure(tmp_path / "p.pdb", FLAGS)
    modes, xyz, lam = st.anm(n_modes, 0.5, 10, 30)
    m2, x2, l2 = anm_oracle.anm(st.xyz, names, first, n_modes, 0.5, 10, 30)
    assert np.array_equal(xyz, x2)
    assert np.allclose(lam, l2, rtol=1e-10, atol=0)
    assert np.abs(modes - _align_signs(modes, m2)).max() <= 1e-8 * np.abs(m2).max()


@pytest.mark.gpu
def test_anm_errors(tmp_path):
    protein_pdb(tmp_path / "p.pdb", 3, 1)
    st = sd.Structure(tmp_path / "p.pdb", FLAGS)
    with pytest.raises(sd.SparkleError):
        st.anm(10, 0.5, 1, 1)  # 16 eigenpairs of a 9 x 9 Hessian
    with pytest.raises(sd.SparkleError):
        st.anm(0, 0.5, 1, 1)
    # a residue without CA: the reference would map residues onto the wrong nodes
    protein_pdb(tmp_path / "q.pdb", 30, 2)
    text = [ln for ln in (tmp_path / "q.pdb").read_text().splitlines()
            if not (ln[12:16] == " CA " and ln[22:26] == "   5")]
    (tmp_path / "q.pdb").write_text("\n".join(text) + "\n")
    with pytest.raises(sd.SparkleError):
        sd.Structure(tmp_path / "q.pdb", FLAGS).anm(5, 0.5, 1, 1)
