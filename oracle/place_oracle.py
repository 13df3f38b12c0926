"""ORACLE (test infrastructure only; never imported by the product): a numpy restatement of the
reference's swarm placement, calculate_start_pos (source/dock/src/cal_anm.cc:775-990) with
calculate_surface_point (:541-774), select_surface (:991-1018), points_on_sphere (:1101-1113) and
kmeans_init_centers3 / run_kmeans3 (source/dock/src/kmeans.cc:126-241), with the C++ library
draws it uses restated: std::mt19937 (Matsumoto and Nishimura's MT19937, init_genrand seeding),
std::uniform_int_distribution over it (libstdc++: Lemire's multiply-and-reject with 64-bit
products), std::uniform_real_distribution<float> and <double> (generate_canonical: one 32-bit draw
over 2^32 in float; two draws, low word first, over 2^64 in double; both clamped below 1), and
std::normal_distribution over minstd_rand0 (anm_oracle).

Every sum the reference forms sequentially is formed sequentially here (np.cumsum, np.bincount),
every distance as sqrt(((dx^2 + dy^2) + dz^2)), so the result is meant to equal the reference's
to the bit.
"""
import math

import numpy as np

from anm_oracle import _MinstdRand0, _NormalDistribution

SURFACE_RESIDUES = ("ARG", "ASN", "ASP", "ASX", "CSO", "GLN", "GLU", "GLX", "GLY", "HID", "HIE", "HIP", "IS",
                    "HSD", "HSE", "HSP", "LYS", "PHD", "PRO", "PTR", "SEP", "SER", "THR", "TPO", "TYR", "HIS")
SPHERES_PER_CENTROID = 100
SURFACE_CUTOFF = 3.0
NEIGHBOUR_CENTROID = 20.0
DEFAULT_SWARM_RADIUS = 10.0
KMEANS_SEED = 324324
PI = 3.14159265358979323846


class MT19937:
    """std::mt19937: init_genrand seeding, 32-bit tempered outputs."""

    def __init__(self, seed):
        self.mt = [0] * 624
        self.mt[0] = seed & 0xFFFFFFFF
        for i in range(1, 624):
            self.mt[i] = (1812433253 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.i = 624

    def _twist(self):
        mt = self.mt
        for k in range(624):
            y = (mt[k] & 0x80000000) | (mt[(k + 1) % 624] & 0x7FFFFFFF)
            mt[k] = mt[(k + 397) % 624] ^ (y >> 1) ^ (0x9908B0DF if y & 1 else 0)
        self.i = 0

    def __call__(self):
        if self.i >= 624:
            self._twist()
        y = self.mt[self.i]
        self.i += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF


def uniform_int(g, lo, hi):
    """std::uniform_int_distribution<int>(lo, hi) over a 32-bit engine (Lemire's method)."""
    rng = hi - lo + 1
    prod = g() * rng
    low = prod & 0xFFFFFFFF
    if low < rng:
        threshold = ((1 << 32) - rng) % rng
        while low < threshold:
            prod = g() * rng
            low = prod & 0xFFFFFFFF
    return (prod >> 32) + lo


def uniform_float(g):
    """std::uniform_real_distribution<float>(0, 1), widened to double."""
    r = np.float32(g()) / np.float32(4294967296.0)
    if r >= np.float32(1.0):
        r = np.nextafter(np.float32(1.0), np.float32(0.0))
    return float(r)


def uniform_double(g):
    """std::uniform_real_distribution<double>(0, 1)."""
    s = float(g())
    s += float(g()) * 4294967296.0
    r = s / 18446744073709551616.0
    return r if r < 1.0 else math.nextafter(1.0, 0.0)


def _d2(a, b):
    d = a - b
    return (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]


def kmeans_seed(pts, K):
    """kmeans_init_centers3(center, pts, n, K, 324324)."""
    n = pts.shape[0]
    g = MT19937(KMEANS_SEED)
    first = uniform_int(g, 0, n - 1)
    cent = np.repeat(pts[first][None, :], K, axis=0)
    mind = np.full(n, np.finfo(np.float64).max)
    for k in range(1, K):
        d = np.sqrt(_d2(pts, cent[k - 1]))
        mind = np.where(d < mind, d, mind)
        total = np.cumsum(mind)[-1]
        t0 = total * uniform_float(g)
        chain = np.cumsum(np.concatenate([[t0], -mind]))[1:]  # t - f0, (t - f0) - f1, ...
        hit = np.nonzero(~(chain > 0))[0]
        if hit.size:
            cent[k] = pts[hit[0]]
    return cent


def kmeans_lloyd(pts, cent, iters):
    """run_kmeans3: assignment to the first strictly nearest centre, then the member means."""
    cent = cent.copy()
    K = cent.shape[0]
    prev = None
    for _ in range(iters):
        d = np.sqrt(_d2(cent[None, :, :], pts[:, None, :]))  # Distance3(centre, point)
        d = np.where(np.isnan(d), np.inf, d)
        group = np.argmin(d, axis=1)
        group[~(np.min(d, axis=1) < np.finfo(np.float32).max)] = -1
        if prev is not None and np.array_equal(group, prev):
            break  # the same assignment gives the same centres from here on
        prev = group
        ok = group >= 0
        cnt = np.bincount(group[ok], minlength=K).astype(np.float64)
        with np.errstate(invalid="ignore", divide="ignore"):
            for c in range(3):
                cent[:, c] = np.bincount(group[ok], weights=pts[ok, c], minlength=K) / (1.0 * cnt)
    return cent


def unit_sphere(n=SPHERES_PER_CENTROID):
    inc = PI * (3.0 - math.sqrt(5.0))
    off = 2.0 / n
    out = np.empty((n, 3))
    for i in range(n):
        y = i * off - 1.0 + (off / 2.0)
        r = math.sqrt(1 - y * y)
        phi = i * inc
        out[i] = (math.cos(phi) * r, y, math.sin(phi) * r)
    return out


def swarm_centres(rec_raw, rec_res_names, rec_res_first, rec_translation, lig_raw, n_swarms):
    """calculate_surface_point: swarm centres [n_swarms][3] in the centred receptor frame."""
    rec_raw, lig_raw = np.asarray(rec_raw, np.float64), np.asarray(lig_raw, np.float64)
    K = n_swarms
    diam2 = 0.0
    for i in range(lig_raw.shape[0] - 1):
        diam2 = max(diam2, float(np.max(_d2(lig_raw[i + 1:], lig_raw[i]))))
    diam = math.sqrt(diam2)
    sdist = DEFAULT_SWARM_RADIUS if diam < DEFAULT_SWARM_RADIUS * 2 else diam / 4.0
    idx = [a for r, name in enumerate(rec_res_names) if name in SURFACE_RESIDUES
           for a in range(rec_res_first[r], rec_res_first[r + 1])]
    surf = rec_raw[idx]
    if surf.shape[0] <= K:
        raise ValueError("not more surface atoms than swarms")
    cent = kmeans_lloyd(surf, kmeans_seed(surf, K), 100)
    if not np.all(np.isfinite(cent)):
        raise ValueError("empty surface cluster")
    samp = (unit_sphere()[None, :, :] * sdist + cent[:, None, :]).reshape(-1, 3)  # [K * 100][3]
    owner = np.repeat(np.arange(K), SPHERES_PER_CENTROID)
    near_c = np.sqrt(_d2(cent[:, None, :], cent[None, :, :])) <= NEIGHBOUR_CENTROID
    np.fill_diagonal(near_c, False)
    keep = np.ones(samp.shape[0], bool)
    for j in range(K):
        rows = near_c[owner, j]
        keep &= ~(rows & (np.sqrt(_d2(samp, cent[j])) <= sdist))
    for a0 in range(0, rec_raw.shape[0], 512):
        blk = rec_raw[a0:a0 + 512]
        keep &= ~np.any(np.sqrt(_d2(samp[:, None, :], blk[None, :, :])) <= SURFACE_CUTOFF, axis=1)
    kept = samp[keep]
    if kept.shape[0] <= K:
        raise ValueError("not more kept sphere points than swarms")
    cent = kmeans_lloyd(kept, kmeans_seed(kept, K), 500)
    if not np.all(np.isfinite(cent)):
        raise ValueError("empty swarm cluster")
    return cent + np.asarray(rec_translation, np.float64)


def start_poses(centres, n_glowworms, n_modes_rec, n_modes_lig, use_anm, seed, anm_seed,
                swarm_radius=DEFAULT_SWARM_RADIUS, rank=0):
    """calculate_start_pos's sampling: poses [swarms][glowworms][7 + modes]."""
    S = centres.shape[0]
    g = MT19937(seed + rank)
    ng, nd = _MinstdRand0(anm_seed), _NormalDistribution()
    pl = 7 + n_modes_rec + n_modes_lig
    out = np.zeros((S, n_glowworms, pl))
    r2 = swarm_radius * swarm_radius
    for i in range(S):
        for j in range(n_glowworms):
            while True:
                x = (2 * uniform_double(g) - 1) * swarm_radius
                y = (2 * uniform_double(g) - 1) * swarm_radius
                z = (2 * uniform_double(g) - 1) * swarm_radius
                if x * x + y * y + z * z <= r2:
                    break
            p = out[i, j]
            p[0], p[1], p[2] = centres[i, 0] + x, centres[i, 1] + y, centres[i, 2] + z
            u1, u2, u3 = uniform_double(g), uniform_double(g), uniform_double(g)
            p[3] = math.sqrt(1 - u1) * math.sin(2 * PI * u2)
            p[4] = math.sqrt(1 - u1) * math.cos(2 * PI * u2)
            p[5] = math.sqrt(u1) * math.sin(2 * PI * u3)
            p[6] = math.sqrt(u1) * math.cos(2 * PI * u3)
            if use_anm:
                for m in range(n_modes_rec + n_modes_lig):
                    p[7 + m] = nd(ng)
    return out


def read_pdb(path):
    """The few fields the placement reads, for the simple PDB files the tests write (ATOM lines,
    no alternates, hydrogens or waters): raw coordinates through float, residue names and first
    atoms, and the centring translation as init_center_translate forms it (the negated mean of
    the non-hydrogen atoms, summed in file order)."""
    xyz, names, first, last = [], [], [], None
    with open(path) as f:
        for ln in f:
            if not ln.startswith("ATOM"):
                continue
            key = (ln[17:21].strip(), int(ln[22:26]), ln[26])
            if key != last:
                first.append(len(xyz))
                names.append(key[0])
                last = key
            xyz.append([float(np.float32(float(ln[30 + 8 * k:38 + 8 * k]))) for k in range(3)])
    first.append(len(xyz))
    xyz = np.array(xyz)
    t = [0.0, 0.0, 0.0]
    for a in xyz:
        for k in range(3):
            t[k] += a[k]
    return xyz, names, first, [-1 * t[k] / len(xyz) for k in range(3)]
