"""ORACLE (test infrastructure only; never imported by the product): a numpy restatement of the
reference's ANM normal modes, cal_anm (source/dock/src/cal_anm.cc:61-219) with build_hessian1D
(:307-360), calModes (:403-514) and norm (:516-540).  The eigensolver is numpy's LAPACK eigh in
place of the reference's cuSOLVER syevd (source/dock/src/cuda/cal_anm.cu:28-91), so eigenvectors
agree with the GPU path to rounding and up to sign; the Hessian and the extent draws are exact.
"""
import math

import numpy as np

CUTOFF = 15.0
GAMMA = 1.0
ZERO_EIGENVALUE = 1e-6
EXPECTED_ZEROS = 6
ANM_SEED = 324324  # cal_anm.cc:171, fixed whatever the setup's anm_seed


def recentre(xyz):
    """norm (cal_anm.cc:516-540): subtract the mean of all atoms, each axis summed in file order."""
    xyz = np.array(xyz, dtype=np.float64)
    m = [0.0, 0.0, 0.0]
    for i in range(xyz.shape[0]):
        for d in range(3):
            m[d] += xyz[i, d]
    return xyz - np.array([m[d] / xyz.shape[0] for d in range(3)])


def nodes_of(xyz, names):
    """Node atoms: CA in file order, else C4 (cal_anm.cc:66-74)."""
    for nm in ("CA", "C4"):
        idx = [i for i, n in enumerate(names) if n == nm]
        if idx:
            return xyz[idx]
    raise ValueError("no CA or C4 atoms")


def hessian(nodes, cutoff=CUTOFF, gamma=GAMMA):
    """build_hessian1D: -g d d^T / |d|^2 off the diagonal for pairs within the cutoff; each
    diagonal block minus its row's blocks, subtracted in increasing partner order (the reference's
    pair loop), so the matrix is the reference's to the bit."""
    n = nodes.shape[0]
    H = np.zeros((3 * n, 3 * n))
    diag = np.zeros((n, 3, 3))
    for p in range(n):  # partner p of every node i, in increasing p
        lo = np.minimum(np.arange(n), p)
        hi = np.maximum(np.arange(n), p)
        d = nodes[hi] - nodes[lo]  # the pair as the reference orders it (j - i, i < j)
        dist2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        ok = (np.arange(n) != p) & ~(dist2 > cutoff * cutoff)
        with np.errstate(divide="ignore", invalid="ignore"):
            se = d[:, :, None] * d[:, None, :] * (-gamma / dist2)[:, None, None]
        se[~ok] = 0.0
        diag = np.where(ok[:, None, None], diag - se, diag)
        for i in np.nonzero(ok)[0]:
            H[3 * i:3 * i + 3, 3 * p:3 * p + 3] = se[i]
    for i in range(n):
        H[3 * i:3 * i + 3, 3 * i:3 * i + 3] = diag[i]
    return H


class _MinstdRand0:
    """std::default_random_engine of libstdc++: minstd_rand0, x <- 16807 x mod (2^31 - 1)."""

    def __init__(self, seed):
        s = seed % 2147483647
        self.x = 1 if s == 0 else s

    def __call__(self):
        self.x = (self.x * 16807) % 2147483647
        return self.x


class _NormalDistribution:
    """std::normal_distribution<double>(0, 1) of libstdc++: Marsaglia's polar method on two
    uniforms, the second value of each accepted pair kept for the next call; the uniforms are
    std::generate_canonical<double, 53> over minstd_rand0 (two draws, (a - 1) + (b - 1) R over R^2,
    R = 2^31 - 2, clamped below 1)."""

    R = 2147483646.0

    def __init__(self):
        self.saved = None

    def _canonical(self, g):
        s = float(g() - 1)
        s += float(g() - 1) * self.R
        r = s / (self.R * self.R)
        return r if r < 1.0 else math.nextafter(1.0, 0.0)

    def __call__(self, g):
        if self.saved is not None:
            v, self.saved = self.saved, None
            return v
        while True:
            x = 2.0 * self._canonical(g) - 1.0
            y = 2.0 * self._canonical(g) - 1.0
            r2 = x * x + y * y
            if r2 <= 1.0 and r2 != 0.0:
                break
        mult = math.sqrt(-2.0 * math.log(r2) / r2)
        self.saved = x * mult
        return y * mult


def extent_coef(eigvals, n_draws):
    """Mean over n_draws extent vectors of sqrt(sum_m v_m^2 / lambda_m), v ~ N(0, 1) drawn in
    order (cal_anm.cc:166-182; its OpenMP loop has no reduction, this is its one-thread value)."""
    g, nd = _MinstdRand0(ANM_SEED), _NormalDistribution()
    coef = 0.0
    for _ in range(n_draws):
        s = 0.0
        for lam in eigvals:
            v = nd(g)
            s += v * v * (1.0 / lam)
        coef += math.sqrt(s)
    return coef / n_draws


def anm(xyz, names, residue_first, n_modes, rmsd, n_swarms, n_glowworms):
    """cal_anm on one structure: returns (modes [n_modes][n_atoms][3], re-centred coordinates,
    eigenvalues [n_modes])."""
    xyz = recentre(xyz)
    nodes = nodes_of(xyz, names)
    H = hessian(nodes)
    w, v = np.linalg.eigh(H)
    length = n_modes + EXPECTED_ZEROS
    w, v = w[:length], v[:, :length]
    nz = int(np.sum(w < ZERO_EIGENVALUE))
    lam, vec = w[nz:nz + n_modes], v[:, nz:nz + n_modes]  # [dof][n_modes]
    na = xyz.shape[0]
    ev = np.empty((na * 3, n_modes))
    for r in range(len(residue_first) - 1):  # every atom of residue r takes node r's rows
        for a in range(residue_first[r], residue_first[r + 1]):
            ev[3 * a:3 * a + 3] = vec[3 * r:3 * r + 3]
    ev /= np.sqrt(np.sum(ev * ev, axis=0))
    coef = extent_coef(lam, n_swarms * n_glowworms)
    ev *= math.sqrt(na) * rmsd / coef * np.sqrt(1.0 / lam)
    return ev.T.reshape(n_modes, na, 3), xyz, lam
