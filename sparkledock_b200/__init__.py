"""sparkledock_b200 — B200-native glowworm swarm optimisation (GSO) docking step.

Python view of the C ABI in include/sparkle_b200.h (libsparkle_b200.so).  It mirrors the
reference's hot-path boundary, prepare_gso_tasks / cal_gso_tasks_gpu
(source/dock/include/prepare_gso_tasks.h:8-26): a set of complexes with swarms of
glowworms, the SoA glowworm state, the reference's random draws, one call per GSO step.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import (SD_PDB_NOH, SD_PDB_NOW, SD_PDB_NOXT, SD_PREC_FP64, SD_PREC_FP64_REF,  # noqa: F401
                   SD_PREC_MIXED, SD_SCORING_DFIRE, SD_SCORING_PYDOCK, SparkleError, check, dptr, iptr)

__all__ = ["SyntheticComplex", "Structure", "synthetic_tables", "synthetic_protein_pdb", "place_swarms",
           "write_pose_pdb", "reference_point", "write_checkpoint", "read_checkpoint", "gso_draws", "mixed_variant_count", "GsoParams", "Docking",
           "SD_PREC_FP64_REF", "SD_PREC_FP64", "SD_PREC_MIXED", "SD_SCORING_DFIRE",
           "SD_SCORING_PYDOCK", "SparkleError", "device_count"]


def device_count() -> int:
    n = C.c_int(0)
    check(_abi.lib().sd_device_count(C.byref(n)), "sd_device_count")
    return n.value


def mixed_variant_count() -> int:
    """Number of compiled variants of the mixed-precision DFIRE kernel (autotuner candidates)."""
    return int(_abi.lib().sd_mixed_variant_count())


def gso_draws(seed: int, n_swarms: int, n_steps: int, n_glowworms: int) -> np.ndarray:
    """The reference's draws u[s][t][g] (std::mt19937(seed), uniform_real_distribution(0,1))."""
    out = np.empty((n_swarms, n_steps, n_glowworms), np.float64)
    check(_abi.lib().sd_gso_draws(seed, n_swarms, n_steps, n_glowworms, dptr(out)), "sd_gso_draws")
    return out


def synthetic_tables(seed: int = 2024):
    """Seeded N(0,1) DFIRE table [168*168*20] and a 20-type LJ (eps, sigma) table."""
    t = np.empty(_abi.SD_DFIRE_TYPES * _abi.SD_DFIRE_TYPES * _abi.SD_DFIRE_BINS, np.float64)
    e = np.empty(_abi.SD_LJ_TYPES, np.float64)
    s = np.empty(_abi.SD_LJ_TYPES, np.float64)
    check(_abi.lib().sd_synth_tables(seed, dptr(t), dptr(e), dptr(s)), "sd_synth_tables")
    return t, e, s


class SyntheticComplex:
    """A seeded synthetic receptor/ligand pair with swarms and starting poses."""

    def __init__(self, n_rec, n_lig, n_swarms, n_glowworms=200, n_modes_rec=10, n_modes_lig=10, seed=1):
        spec = _abi.SynthSpec(n_rec, n_lig, n_swarms, n_glowworms, n_modes_rec, n_modes_lig, seed)
        nbytes = C.c_longlong(0)
        L = _abi.lib()
        check(L.sd_synth_buffer_size(C.byref(spec), C.byref(nbytes)), "sd_synth_buffer_size")
        self._buf = np.zeros(nbytes.value, np.uint8)
        self.desc = _abi.ComplexDesc()
        poses = _abi._dp()
        check(L.sd_synth_generate(C.byref(spec), self._buf.ctypes.data_as(C.c_void_p), C.byref(self.desc),
                                  C.byref(poses)), "sd_synth_generate")
        self.spec = spec
        self.n_rec, self.n_lig = n_rec, n_lig
        self.n_swarms, self.n_glowworms = n_swarms, n_glowworms
        self.n_modes_rec, self.n_modes_lig = n_modes_rec, n_modes_lig
        self.pose_len = 7 + n_modes_rec + n_modes_lig
        d = self.desc

        base = self._buf.ctypes.data

        def view(ptr, shape, dtype):
            # a slice of self._buf, so every array keeps the buffer alive after the complex is gone
            n = int(np.prod(shape))
            if n == 0:
                return np.zeros(shape, dtype)
            item = np.dtype(dtype).itemsize
            off = C.cast(ptr, C.c_void_p).value - base
            if off < 0 or off + n * item > self._buf.nbytes or off % item:
                raise SparkleError(_abi.SD_ERR_ARG, "sd_synth_generate: an array outside its buffer")
            return self._buf[off:off + n * item].view(dtype).reshape(shape)

        self.rec_xyz = view(d.rec_xyz, (n_rec, 3), np.float64)
        self.lig_xyz = view(d.lig_xyz, (n_lig, 3), np.float64)
        self.rec_mask = view(d.rec_mask, (n_rec,), np.int32)
        self.lig_mask = view(d.lig_mask, (n_lig,), np.int32)
        self.rec_modes = view(d.rec_modes, (n_modes_rec, n_rec, 3), np.float64)
        self.lig_modes = view(d.lig_modes, (n_modes_lig, n_lig, 3), np.float64)
        self.rec_type = view(d.rec_dfire_type, (n_rec,), np.int32)
        self.lig_type = view(d.lig_dfire_type, (n_lig,), np.int32)
        self.rec_charge = view(d.rec_charge, (n_rec,), np.float64)
        self.lig_charge = view(d.lig_charge, (n_lig,), np.float64)
        self.rec_lj = view(d.rec_lj_type, (n_rec,), np.int32)
        self.lig_lj = view(d.lig_lj_type, (n_lig,), np.int32)
        self.poses = view(poses, (n_swarms, n_glowworms, self.pose_len), np.float64)

    @property
    def lig_ref(self) -> np.ndarray:
        """The ligand reference point of the descriptor (a copy; assign to change it)."""
        return np.array(list(self.desc.lig_ref_point), np.float64)

    @lig_ref.setter
    def lig_ref(self, v) -> None:
        for k in range(3):
            self.desc.lig_ref_point[k] = float(v[k])


class Structure:
    """A structure read from a PDB file as the reference's setup reads it (first MODEL, centred
    coordinates, normal-mode mask, DFIRE atom types, CA/P backbone flags); flags are
    SD_PDB_NOXT | SD_PDB_NOH | SD_PDB_NOW (setup.json noxt / noh / now)."""

    def __init__(self, path: str, flags: int = 0):
        self.path, self.flags = str(path), flags
        h = C.c_void_p()
        check(_abi.lib().sd_structure_load(str(path).encode(), flags, C.byref(h)), "sd_structure_load")
        try:
            n, nr = C.c_int(), C.c_int()
            check(_abi.lib().sd_structure_info(h, C.byref(n), C.byref(nr)), "sd_structure_info")
            self.n_atoms, self.n_residues = n.value, nr.value
            self.xyz = np.empty((self.n_atoms, 3))
            self.nm_mask = np.empty(self.n_atoms, np.int32)
            self.dfire_type = np.empty(self.n_atoms, np.int32)
            self.backbone = np.empty(self.n_atoms, np.int32)
            self.translation = np.empty(3)
            check(_abi.lib().sd_structure_arrays(h, dptr(self.xyz), iptr(self.nm_mask), iptr(self.dfire_type),
                                                 iptr(self.backbone), dptr(self.translation)), "sd_structure_arrays")
        finally:
            _abi.lib().sd_structure_free(h)

    def anm(self, n_modes: int, rmsd: float, n_swarms: int, n_glowworms: int, device: int = 0):
        """Normal modes as the reference's setup computes them (sd_anm): modes
        [n_modes][n_atoms][3], the re-centred coordinates they belong to [n_atoms][3] and the
        eigenvalues [n_modes]."""
        h = C.c_void_p()
        check(_abi.lib().sd_structure_load(self.path.encode(), self.flags, C.byref(h)), "sd_structure_load")
        try:
            modes = np.empty((n_modes, self.n_atoms, 3))
            xyz = np.empty((self.n_atoms, 3))
            lam = np.empty(n_modes)
            check(_abi.lib().sd_anm(h, n_modes, rmsd, n_swarms, n_glowworms, device, dptr(modes), dptr(xyz),
                                    dptr(lam)), "sd_anm")
        finally:
            _abi.lib().sd_structure_free(h)
        return modes, xyz, lam


def reference_point(xyz) -> np.ndarray:
    """The ligand reference point (sd_reference_point: Khachiyan minimum-volume enclosing
    ellipsoid centre, tolerance 0.01) of coordinates [n][3]."""
    x = np.ascontiguousarray(xyz, np.float64)
    out = np.empty(3)
    check(_abi.lib().sd_reference_point(dptr(x), x.shape[0], dptr(out)), "sd_reference_point")
    return out


def write_pose_pdb(path, receptor: Structure, rec_xyz, ligand: Structure = None, lig_xyz=None) -> None:
    """Write one pose as the reference writes lightdock_<g>.pdb (sd_write_pose_pdb): the
    receptor's atoms at rec_xyz [n_rec][3], then the ligand's at lig_xyz."""
    lib = _abi.lib()
    hr, hl = C.c_void_p(), C.c_void_p()
    check(lib.sd_structure_load(receptor.path.encode(), receptor.flags, C.byref(hr)), "sd_structure_load")
    try:
        rx = np.ascontiguousarray(rec_xyz, np.float64)
        lx = None
        if ligand is not None:
            check(lib.sd_structure_load(ligand.path.encode(), ligand.flags, C.byref(hl)), "sd_structure_load")
            lx = np.ascontiguousarray(lig_xyz, np.float64)
        if rx.shape != (receptor.n_atoms, 3) or (lx is not None and lx.shape != (ligand.n_atoms, 3)):
            raise ValueError("coordinates must be [n_atoms][3] for each structure")
        check(lib.sd_write_pose_pdb(str(path).encode(), hr, dptr(rx), hl if ligand is not None else None,
                                    dptr(lx) if lx is not None else None), "sd_write_pose_pdb")
    finally:
        lib.sd_structure_free(hr)
        if hl.value:
            lib.sd_structure_free(hl)


def place_swarms(receptor: Structure, ligand: Structure, n_swarms: int, n_glowworms: int, n_modes_rec: int = 0,
                 n_modes_lig: int = 0, use_anm: bool = True, starting_points_seed: int = 324324,
                 anm_seed: int = 324324, swarm_radius: float = 10.0, rank: int = 0, device: int = 0):
    """Swarm centres [n_swarms][3] (centred receptor frame) and starting poses
    [n_swarms][n_glowworms][7 + modes] as the reference's setup places them (sd_place_swarms)."""
    lib = _abi.lib()
    hr, hl = C.c_void_p(), C.c_void_p()
    check(lib.sd_structure_load(receptor.path.encode(), receptor.flags, C.byref(hr)), "sd_structure_load")
    try:
        check(lib.sd_structure_load(ligand.path.encode(), ligand.flags, C.byref(hl)), "sd_structure_load")
        centers = np.empty((n_swarms, 3))
        poses = np.empty((n_swarms, n_glowworms, 7 + n_modes_rec + n_modes_lig))
        check(lib.sd_place_swarms(hr, hl, n_swarms, n_glowworms, n_modes_rec, n_modes_lig, int(use_anm),
                                  starting_points_seed, anm_seed, swarm_radius, rank, device, dptr(centers),
                                  dptr(poses)), "sd_place_swarms")
    finally:
        lib.sd_structure_free(hr)
        if hl.value:
            lib.sd_structure_free(hl)
    return centers, poses


def GsoParams(**kw) -> _abi.GsoParams:
    p = _abi.GsoParams()
    _abi.lib().sd_gso_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@dataclass
class State:
    pos: np.ndarray
    scoring: np.ndarray
    luciferin: np.ndarray
    vision_range: np.ndarray
    step: np.ndarray
    moved: np.ndarray
    nnei_len: np.ndarray
    select: np.ndarray
    ligand_reference_pose: np.ndarray

    @staticmethod
    def empty(S, G, pl):
        return State(np.zeros((S, G, pl)), np.zeros((S, G)), np.zeros((S, G)), np.zeros((S, G)),
                     np.zeros((S, G), np.int32), np.zeros((S, G), np.int32), np.zeros((S, G), np.int32),
                     np.zeros((S, G), np.int32), np.zeros((S, G, 3)))

    def as_c(self) -> _abi.SwarmState:
        return _abi.SwarmState(dptr(self.pos), dptr(self.scoring), dptr(self.luciferin), dptr(self.vision_range),
                               iptr(self.step), iptr(self.moved), iptr(self.nnei_len), iptr(self.select),
                               dptr(self.ligand_reference_pose))

    def copy(self) -> "State":
        return State(*(np.array(getattr(self, f)) for f in self.__dataclass_fields__))


def write_checkpoint(path, state: State, steps_done: int, steps_total: int = 0) -> None:
    """Write a GSO state, the steps taken and the steps the run was started with (0: not given) to
    a checkpoint file (sd_write_checkpoint)."""
    S, G, pl = state.pos.shape
    cs = state.as_c()
    check(_abi.lib().sd_write_checkpoint(str(path).encode(), S, G, pl, steps_done, steps_total, C.byref(cs)),
          "sd_write_checkpoint")


def read_checkpoint(path):
    """(State, steps_done, steps_total) from a checkpoint file (sd_read_checkpoint)."""
    S, G, pl, done, total = C.c_int(), C.c_int(), C.c_int(), C.c_longlong(), C.c_longlong()
    check(_abi.lib().sd_checkpoint_info(str(path).encode(), C.byref(S), C.byref(G), C.byref(pl), C.byref(done),
                                        C.byref(total)), "sd_checkpoint_info")
    st = State.empty(S.value, G.value, pl.value)
    cs = st.as_c()
    check(_abi.lib().sd_read_checkpoint(str(path).encode(), S.value, G.value, pl.value, C.byref(done),
                                        C.byref(total), C.byref(cs)), "sd_read_checkpoint")
    return st, done.value, total.value


class Docking:
    """A context on one GPU holding complexes, their GSO state and the step graph."""

    def __init__(self, complexes, tables, params=None, scoring=SD_SCORING_DFIRE, precision=SD_PREC_MIXED,
                 device=0):
        self._complexes = list(complexes)
        descs = (_abi.ComplexDesc * len(self._complexes))(*[c.desc for c in self._complexes])
        self._tables_np = tables
        t = _abi.Tables(dptr(tables[0]), dptr(tables[1]), dptr(tables[2]))
        self._params = params if params is not None else GsoParams()
        ctx = C.c_void_p()
        check(_abi.lib().sd_ctx_create(descs, len(self._complexes), C.byref(t), C.byref(self._params), scoring,
                                       precision, device, C.byref(ctx)), "sd_ctx_create")
        self._ctx = ctx

    def close(self):
        if getattr(self, "_ctx", None):
            _abi.lib().sd_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(_abi.lib().sd_ctx_stream(self._ctx, C.byref(s)), "sd_ctx_stream")
        return s.value or 0

    def init_state(self, ci: int, pos: np.ndarray):
        pos = np.ascontiguousarray(pos, np.float64)
        check(_abi.lib().sd_init_state(self._ctx, ci, dptr(pos)), "sd_init_state")

    def set_state(self, ci: int, st: State):
        cs = st.as_c()
        check(_abi.lib().sd_set_state(self._ctx, ci, C.byref(cs)), "sd_set_state")

    def get_state(self, ci: int) -> State:
        c = self._complexes[ci]
        st = State.empty(c.n_swarms, c.n_glowworms, c.pose_len)
        cs = st.as_c()
        check(_abi.lib().sd_get_state(self._ctx, ci, C.byref(cs)), "sd_get_state")
        return st

    def set_draws(self, ci: int, u: np.ndarray):
        u = np.ascontiguousarray(u, np.float64)
        check(_abi.lib().sd_set_draws(self._ctx, ci, dptr(u), u.shape[1]), "sd_set_draws")

    def step(self, n: int = 1, sync: bool = True):
        check(_abi.lib().sd_step(self._ctx, n, 1 if sync else 0), "sd_step")

    def tuning(self) -> dict:
        v, w, mb = C.c_int(), C.c_int(), C.c_int()
        n = mixed_variant_count()
        ms = np.zeros(n)
        check(_abi.lib().sd_get_tuning(self._ctx, C.byref(v), C.byref(w), C.byref(mb), dptr(ms), n), "sd_get_tuning")
        return {"variant": v.value, "warps": w.value, "min_blocks": mb.value, "ms": [float(x) for x in ms]}

    def cluster(self, ci: int, rec_backbone, lig_backbone) -> dict:
        """BSAS clustering of the current poses of every swarm of complex ci (sd_cluster)."""
        c = self._complexes[ci]
        S, G = c.n_swarms, c.n_glowworms
        rb = np.ascontiguousarray(rec_backbone, np.int32)
        lb = np.ascontiguousarray(lig_backbone, np.int32)
        ncl = np.empty(S, np.int32)
        rep, size, member = (np.empty((S, G), np.int32) for _ in range(3))
        check(_abi.lib().sd_cluster(self._ctx, ci, iptr(rb), iptr(lb), iptr(ncl), iptr(rep), iptr(size),
                                    iptr(member)), "sd_cluster")
        return {"n_clusters": ncl, "rep": rep, "size": size, "member": member}

    def materialise(self, ci: int, poses):
        """Every atom of the chosen glowworms (index swarm * n_glowworms + glowworm) of complex ci at
        their current poses (sd_materialise_poses): receptor [n][n_rec][3], ligand [n][n_lig][3]."""
        c = self._complexes[ci]
        idx = np.ascontiguousarray(poses, np.int32).ravel()
        rec = np.empty((idx.size, c.n_rec, 3))
        lig = np.empty((idx.size, c.n_lig, 3))
        check(_abi.lib().sd_materialise_poses(self._ctx, ci, iptr(idx), idx.size, dptr(rec), dptr(lig)),
              "sd_materialise_poses")
        return rec, lig

    def set_precision(self, precision: int):
        check(_abi.lib().sd_set_precision(self._ctx, precision), "sd_set_precision")

    def stats(self) -> dict:
        s = _abi.Stats()
        check(_abi.lib().sd_get_stats(self._ctx, C.byref(s)), "sd_get_stats")
        return {f: getattr(s, f) for f, _ in _abi.Stats._fields_}

    def score_poses(self, ci: int, poses: np.ndarray, precision: int = SD_PREC_MIXED):
        poses = np.ascontiguousarray(poses, np.float64).reshape(-1, self._complexes[ci].pose_len)
        n = poses.shape[0]
        sc = np.empty(n)
        en = np.empty(n)
        check(_abi.lib().sd_score_poses(self._ctx, ci, dptr(poses), n, precision, dptr(sc), dptr(en)),
              "sd_score_poses")
        return sc, en

    def dfire_bins(self, ci: int, pose: np.ndarray, precision: int = SD_PREC_MIXED) -> np.ndarray:
        c = self._complexes[ci]
        pose = np.ascontiguousarray(pose, np.float64)
        out = np.empty((c.n_rec, c.n_lig), np.int32)
        check(_abi.lib().sd_dfire_bins(self._ctx, ci, dptr(pose), precision, iptr(out)), "sd_dfire_bins")
        return out

    def refine(self, ci: int, poses: np.ndarray, iters: int = 50, step: float = 0.5,
               precision: int = SD_PREC_MIXED):
        """Post-GSO refinement on the pyDock-style energy; returns (poses, E_before, E_after),
        FP64 energies, never increasing."""
        c = self._complexes[ci]
        p = np.array(poses, np.float64).reshape(-1, c.pose_len).copy()
        n = p.shape[0]
        e0 = np.empty(n)
        e1 = np.empty(n)
        check(_abi.lib().sd_refine_poses(self._ctx, ci, dptr(p), n, iters, step, precision, dptr(e0), dptr(e1)),
              "sd_refine_poses")
        return p, e0, e1

    def pydock_grad(self, ci: int, poses: np.ndarray, precision: int = SD_PREC_MIXED):
        c = self._complexes[ci]
        poses = np.ascontiguousarray(poses, np.float64).reshape(-1, c.pose_len)
        n = poses.shape[0]
        e = np.empty(n)
        g = np.empty((n, 6 + c.n_modes_rec + c.n_modes_lig))
        check(_abi.lib().sd_pydock_grad(self._ctx, ci, dptr(poses), n, precision, dptr(e), dptr(g)),
              "sd_pydock_grad")
        return e, g


def synthetic_protein_pdb(path, n_res: int, seed: int):
    """Write a PDB file of a compact synthetic chain of n_res glycines and alanines (N, CA, C, O
    [, CB]; every third residue an alanine): CA steps of 3.8 A inside a sphere, no two CA closer
    than 3.4 A, seeded.  A stand-in protein for tests and benchmarks of the setup stages (reader,
    ANM, swarm placement).  Returns (atom names, first atom of each residue)."""
    rng = np.random.default_rng(seed)
    radius = 2.6 * n_res ** (1.0 / 3.0) + 6.0
    ca = [np.zeros(3)]
    while len(ca) < n_res:
        step = rng.normal(size=3)
        p = ca[-1] + step * (3.8 / np.linalg.norm(step))
        if np.linalg.norm(p) > radius or np.min(np.linalg.norm(np.array(ca) - p, axis=1)) < 3.4:
            if rng.random() < 0.02:  # back out of a dead end
                ca.pop() if len(ca) > 1 else None
            continue
        ca.append(p)

    def bond(origin, length):
        v = rng.normal(size=3)
        return origin + v * (length / np.linalg.norm(v))

    names, first, lines = [], [], []
    for r, p in enumerate(ca):
        first.append(len(names))
        res = "ALA" if r % 3 == 1 else "GLY"
        c = bond(p, 1.52)
        atoms = [("N", bond(p, 1.46)), ("CA", p), ("C", c), ("O", bond(c, 1.23))]
        if res == "ALA":
            atoms.append(("CB", bond(p, 1.53)))
        for nm, x in atoms:
            names.append(nm)
            lines.append("ATOM  %5d  %-3s %s A%4d    %8.3f%8.3f%8.3f  1.00  0.00\n" %
                         (len(names), nm, res, r + 1, x[0] + 30.0, x[1] - 12.0, x[2] + 5.0))
    first.append(len(names))
    with open(path, "w") as f:
        f.writelines(lines)
        f.write("END\n")
    return names, first
