"""ctypes binding of the ORACLE (oracle/liboracle.so, the C restatement) and of the
reference harness (oracle/_ref/libsdref.so, the reference's own compiled CPU functions).
Test infrastructure only: the product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libsdref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OrSystem(C.Structure):
    _fields_ = [
        ("nr", C.c_int), ("nl", C.c_int), ("nmr", C.c_int), ("nml", C.c_int), ("S", C.c_int), ("G", C.c_int),
        ("rec_xyz", _dp), ("lig_xyz", _dp), ("rec_mask", _ip), ("lig_mask", _ip),
        ("rec_modes", _dp), ("lig_modes", _dp), ("rec_type", _ip), ("lig_type", _ip),
        ("table", _dp), ("lig_ref", C.c_double * 3),
        ("rec_charge", _dp), ("lig_charge", _dp), ("rec_lj", _ip), ("lig_lj", _ip),
        ("lj_eps", _dp), ("lj_sigma", _dp),
        ("rho", C.c_double), ("gamma", C.c_double), ("beta", C.c_double), ("max_vision", C.c_double),
        ("max_neighbors", C.c_int),
        ("step_t", C.c_double), ("step_r", C.c_double), ("step_nm", C.c_double),
        ("scoring", C.c_int), ("cr_math", C.c_int),
    ]


class OrState(C.Structure):
    _fields_ = [("pos", _dp), ("scoring", _dp), ("luciferin", _dp), ("vision", _dp), ("step", _ip),
                ("moved", _ip), ("nnei", _ip), ("select", _ip), ("ref", _dp)]


class OrCounts(C.Structure):
    _fields_ = [(n, C.c_longlong) for n in ("scored", "d2_zero", "d2_cutoff", "u_zero", "shortfall")]


class OrSynthOut(C.Structure):
    _fields_ = [(n, _dp) for n in ("rec_xyz", "lig_xyz", "rec_modes", "lig_modes", "rec_charge", "lig_charge",
                                   "poses")] + \
               [(n, _ip) for n in ("rec_mask", "lig_mask", "rec_type", "lig_type", "rec_lj", "lig_lj")] + \
               [("lig_ref", C.c_double * 3)]


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


_oracle = None
_ref = None


def oracle():
    global _oracle
    if _oracle is None:
        L = C.CDLL(ORACLE_SO)
        L.or_gso_draws.argtypes = [C.c_uint, C.c_int, C.c_int, C.c_int, _dp]
        L.or_score_pose.restype = C.c_double
        L.or_score_pose.argtypes = [C.POINTER(OrSystem), _dp, _dp, _dp, _ip, C.POINTER(OrCounts)]
        L.or_score_poses.argtypes = [C.POINTER(OrSystem), _dp, C.c_int, _dp, _dp, C.c_int]
        L.or_receptor_pose.argtypes = [C.POINTER(OrSystem), _dp, _dp]
        L.or_ligand_pose.argtypes = [C.POINTER(OrSystem), _dp, _dp, _dp]
        L.or_gso_step.argtypes = [C.POINTER(OrSystem), C.POINTER(OrState), _dp, _dp, C.POINTER(OrCounts), C.c_int]
        L.or_sin_cr.restype = C.c_double
        L.or_sin_cr.argtypes = [C.c_double]
        L.or_acos_cr.restype = C.c_double
        L.or_acos_cr.argtypes = [C.c_double]
        L.or_slerp.argtypes = [_dp, _dp, C.c_double, C.c_int]
        L.or_key_thresholds.argtypes = [_dp]
        L.or_cluster.argtypes = [C.POINTER(OrSystem), _dp, _dp, _ip, _ip, _ip, _ip, _ip, _ip]
        L.or_pydock_energy.restype = C.c_double
        L.or_pydock_energy.argtypes = [C.POINTER(OrSystem), _dp]
        L.or_pydock_grad.argtypes = [C.POINTER(OrSystem), _dp, _dp]
        L.or_synth_generate.argtypes = [C.c_int] * 6 + [C.c_ulonglong, C.POINTER(OrSynthOut)]
        L.or_synth_tables.argtypes = [C.c_ulonglong, _dp, _dp, _dp]
        L.or_mvee_center.argtypes = [_dp, C.c_int, C.c_double, _dp]
        L.or_crmath_eval.argtypes = [C.c_int, _dp, C.c_longlong, _dp]
        _oracle = L
    return _oracle


class OracleSynthComplex:
    """A seeded synthetic complex built by the oracle's restatement of the product's generator
    (oracle/or_synth.c), bit-identical to sparkledock_b200.SyntheticComplex with the same
    arguments, without loading the product library."""

    def __init__(self, n_rec, n_lig, n_swarms, n_glowworms=200, n_modes_rec=10, n_modes_lig=10, seed=1):
        self.n_rec, self.n_lig = n_rec, n_lig
        self.n_swarms, self.n_glowworms = n_swarms, n_glowworms
        self.n_modes_rec, self.n_modes_lig = n_modes_rec, n_modes_lig
        self.pose_len = 7 + n_modes_rec + n_modes_lig
        self.rec_xyz = np.zeros((n_rec, 3))
        self.lig_xyz = np.zeros((n_lig, 3))
        self.rec_modes = np.zeros((n_modes_rec, n_rec, 3))
        self.lig_modes = np.zeros((n_modes_lig, n_lig, 3))
        self.rec_charge = np.zeros(n_rec)
        self.lig_charge = np.zeros(n_lig)
        self.poses = np.zeros((n_swarms, n_glowworms, self.pose_len))
        self.rec_mask, self.lig_mask = np.zeros(n_rec, np.int32), np.zeros(n_lig, np.int32)
        self.rec_type, self.lig_type = np.zeros(n_rec, np.int32), np.zeros(n_lig, np.int32)
        self.rec_lj, self.lig_lj = np.zeros(n_rec, np.int32), np.zeros(n_lig, np.int32)
        o = OrSynthOut()
        for f in ("rec_xyz", "lig_xyz", "rec_modes", "lig_modes", "rec_charge", "lig_charge", "poses"):
            setattr(o, f, _d(getattr(self, f)))
        for f, a in (("rec_mask", "rec_mask"), ("lig_mask", "lig_mask"), ("rec_type", "rec_type"),
                     ("lig_type", "lig_type"), ("rec_lj", "rec_lj"), ("lig_lj", "lig_lj")):
            setattr(o, f, _i(getattr(self, a)))
        oracle().or_synth_generate(n_rec, n_lig, n_swarms, n_glowworms, n_modes_rec, n_modes_lig, seed, C.byref(o))
        self.lig_ref = np.array(list(o.lig_ref), np.float64)


def oracle_tables(seed: int = 2024):
    """The seeded N(0,1) DFIRE table and LJ table (oracle restatement of the product's)."""
    t = np.empty(168 * 168 * 20)
    e = np.empty(20)
    s = np.empty(20)
    oracle().or_synth_tables(seed, _d(t), _d(e), _d(s))
    return t, e, s


def oracle_draws(seed: int, n_swarms: int, n_steps: int, n_glowworms: int) -> np.ndarray:
    """The reference's draws u[s][t][g] (mt19937 + uniform_real_distribution, oracle restatement)."""
    out = np.empty((n_swarms, n_steps, n_glowworms))
    oracle().or_gso_draws(seed, n_swarms, n_steps, n_glowworms, _d(out))
    return out


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_SO)
        L.ref_score_pose.restype = C.c_double
        L.ref_score_pose.argtypes = [C.POINTER(OrSystem), _dp, _dp, _dp, _dp]
        L.ref_gso_draws.argtypes = [C.c_uint, C.c_int, C.c_int, C.c_int, _dp]
        L.ref_gso_step.restype = C.c_longlong
        L.ref_gso_step.argtypes = [C.POINTER(OrSystem), C.POINTER(OrState), _dp, C.c_int]
        L.ref_slerp.argtypes = [_dp, _dp, C.c_double]
        L.ref_min_volume_ellipsoid.argtypes = [_dp, C.c_int, _dp, _dp]
        L.ref_load_structure.restype = C.c_int
        L.ref_load_structure.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _dp, _ip, _ip, _dp, C.c_int]
        L.ref_write_pose_pdb.restype = C.c_int
        L.ref_write_pose_pdb.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_char_p]
        L.ref_run_cal_gso_tasks_cpu.restype = C.c_int
        L.ref_run_cal_gso_tasks_cpu.argtypes = [C.POINTER(OrSystem), _dp, C.c_int, C.c_char_p, C.c_int]
        _ref = L
    return _ref


class OracleSystem:
    """Holds an OrSystem for one synthetic complex (keeps the arrays alive)."""

    def __init__(self, cx, tables, params=None, n_swarms=None, scoring=0, cr_math=1):
        self.cx = cx
        self.table = np.ascontiguousarray(tables[0])
        self.eps = np.ascontiguousarray(tables[1])
        self.sig = np.ascontiguousarray(tables[2])
        S = cx.n_swarms if n_swarms is None else n_swarms
        s = OrSystem()
        s.nr, s.nl, s.nmr, s.nml, s.S, s.G = cx.n_rec, cx.n_lig, cx.n_modes_rec, cx.n_modes_lig, S, cx.n_glowworms
        self._keep = [np.ascontiguousarray(a) for a in (cx.rec_xyz, cx.lig_xyz, cx.rec_mask, cx.lig_mask,
                                                        cx.rec_modes, cx.lig_modes, cx.rec_type, cx.lig_type,
                                                        cx.rec_charge, cx.lig_charge, cx.rec_lj, cx.lig_lj)]
        k = self._keep
        s.rec_xyz, s.lig_xyz = _d(k[0]), _d(k[1])
        s.rec_mask, s.lig_mask = _i(k[2]), _i(k[3])
        s.rec_modes, s.lig_modes = _d(k[4]), _d(k[5])
        s.rec_type, s.lig_type = _i(k[6]), _i(k[7])
        s.table = _d(self.table)
        for a in range(3):
            s.lig_ref[a] = cx.lig_ref[a]
        s.rec_charge, s.lig_charge = _d(k[8]), _d(k[9])
        s.rec_lj, s.lig_lj = _i(k[10]), _i(k[11])
        s.lj_eps, s.lj_sigma = _d(self.eps), _d(self.sig)
        p = params
        s.rho = p.rho if p else 0.4
        s.gamma = p.gamma if p else 0.6
        s.beta = p.beta if p else 0.08
        s.max_vision = p.max_vision_range if p else 5.0
        s.max_neighbors = p.max_neighbors if p else 5
        s.step_t = p.translation_step if p else 0.5
        s.step_r = p.rotation_step if p else 0.5
        s.step_nm = p.nmodes_step if p else 0.5
        s.scoring = scoring
        s.cr_math = cr_math
        self.s = s
        self.S = S

    @property
    def ptr(self):
        return C.byref(self.s)


class OracleState:
    def __init__(self, S, G, pl, pos0=None, luciferin0=5.0, vision0=0.2):
        self.pos = np.zeros((S, G, pl)) if pos0 is None else np.array(pos0, np.float64).reshape(S, G, pl).copy()
        self.scoring = np.zeros((S, G))
        self.luciferin = np.full((S, G), luciferin0)
        self.vision = np.full((S, G), vision0)
        self.step = np.zeros((S, G), np.int32)
        self.moved = np.zeros((S, G), np.int32)
        self.nnei = np.zeros((S, G), np.int32)
        self.select = np.tile(np.arange(G, dtype=np.int32), (S, 1))
        self.ref = np.zeros((S, G, 3))

    def c(self) -> OrState:
        return OrState(_d(self.pos), _d(self.scoring), _d(self.luciferin), _d(self.vision), _i(self.step),
                       _i(self.moved), _i(self.nnei), _i(self.select), _d(self.ref))

    def copy(self):
        o = OracleState.__new__(OracleState)
        for f in ("pos", "scoring", "luciferin", "vision", "step", "moved", "nnei", "select", "ref"):
            setattr(o, f, np.array(getattr(self, f)))
        return o


def oracle_step(osys: OracleSystem, st: OracleState, u_step: np.ndarray, score_override=None, nthreads=8):
    cnt = OrCounts()
    cs = st.c()
    u = np.ascontiguousarray(u_step, np.float64)
    so = None if score_override is None else _d(np.ascontiguousarray(score_override, np.float64))
    if score_override is not None:
        keep = np.ascontiguousarray(score_override, np.float64)
        so = _d(keep)
    oracle().or_gso_step(osys.ptr, C.byref(cs), _d(u), so, C.byref(cnt), nthreads)
    return cnt


def ref_step(osys: OracleSystem, st: OracleState, u_step: np.ndarray, nthreads=8):
    cs = st.c()
    u = np.ascontiguousarray(u_step, np.float64)
    return ref().ref_gso_step(osys.ptr, C.byref(cs), _d(u), nthreads)


def oracle_scores(osys: OracleSystem, poses: np.ndarray, nthreads=8):
    poses = np.ascontiguousarray(poses, np.float64).reshape(-1, osys.cx.pose_len)
    n = poses.shape[0]
    sc = np.empty(n)
    en = np.empty(n)
    oracle().or_score_poses(osys.ptr, _d(poses), n, _d(sc), _d(en), nthreads)
    return sc, en


def oracle_bins(osys: OracleSystem, pose: np.ndarray):
    pose = np.ascontiguousarray(pose, np.float64)
    bins = np.empty((osys.cx.n_rec, osys.cx.n_lig), np.int32)
    cnt = OrCounts()
    e = C.c_double(0)
    ref = np.zeros(3)
    sc = oracle().or_score_pose(osys.ptr, _d(pose), C.byref(e), _d(ref), _i(bins), C.byref(cnt))
    return bins, sc, e.value, ref, cnt


def ref_structure(path: str, noxt: bool, noh: bool, now: bool, cap: int = 40000):
    """The reference's own setup of one structure (compiled from its sources): centred
    coordinates, normal-mode mask, DFIRE types, translation."""
    xyz = np.empty((cap, 3))
    mask = np.empty(cap, np.int32)
    dfire = np.empty(cap, np.int32)
    tr = np.empty(3)
    n = ref().ref_load_structure(str(path).encode(), int(noxt), int(noh), int(now), _d(xyz), _i(mask), _i(dfire),
                                 _d(tr), cap)
    assert n >= 0
    return xyz[:n].copy(), mask[:n].copy(), dfire[:n].copy(), tr


def oracle_pose_atoms(osys: OracleSystem, pose):
    """Every receptor and ligand atom at one pose (the oracle's exact FP64 transforms)."""
    pose = np.ascontiguousarray(pose, np.float64)
    rec = np.empty((osys.cx.n_rec, 3))
    lig = np.empty((osys.cx.n_lig, 3))
    refp = np.empty(3)
    oracle().or_receptor_pose(osys.ptr, _d(pose), _d(rec))
    oracle().or_ligand_pose(osys.ptr, _d(pose), _d(lig), _d(refp))
    return rec, lig


def oracle_cluster(osys: OracleSystem, pos, scores, rec_bb, lig_bb):
    S, G = osys.S, osys.cx.n_glowworms
    pos = np.ascontiguousarray(pos, np.float64)
    scores = np.ascontiguousarray(scores, np.float64)
    rb = np.ascontiguousarray(rec_bb, np.int32)
    lb = np.ascontiguousarray(lig_bb, np.int32)
    ncl = np.empty(S, np.int32)
    rep, size, member = (np.empty((S, G), np.int32) for _ in range(3))
    oracle().or_cluster(osys.ptr, _d(pos), _d(scores), _i(rb), _i(lb), _i(ncl), _i(rep), _i(size), _i(member))
    return {"n_clusters": ncl, "rep": rep, "size": size, "member": member}
