"""ctypes binding of libsparkle_b200.so (include/sparkle_b200.h).

The library is the product: a GPU call fails loudly when it is missing or was built
without a usable device; there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsparkle_b200.so")

SD_OK, SD_ERR_ARG, SD_ERR_OOM, SD_ERR_CUDA, SD_ERR_TIMEOUT, SD_ERR_NUMERIC, SD_ERR_STATE, SD_ERR_NOTSUP = range(8)
SD_DFIRE_TYPES, SD_DFIRE_BINS, SD_MAX_MODES, SD_LJ_TYPES = 168, 20, 10, 20
SD_SCORING_DFIRE, SD_SCORING_PYDOCK = 0, 1
SD_PREC_FP64_REF, SD_PREC_FP64, SD_PREC_MIXED = 0, 1, 2
SD_PDB_NOXT, SD_PDB_NOH, SD_PDB_NOW = 1, 2, 4

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class ComplexDesc(C.Structure):
    _fields_ = [
        ("n_rec", C.c_int), ("n_lig", C.c_int),
        ("rec_xyz", _dp), ("lig_xyz", _dp),
        ("rec_mask", _ip), ("lig_mask", _ip),
        ("n_modes_rec", C.c_int), ("n_modes_lig", C.c_int),
        ("rec_modes", _dp), ("lig_modes", _dp),
        ("rec_dfire_type", _ip), ("lig_dfire_type", _ip),
        ("rec_charge", _dp), ("lig_charge", _dp),
        ("rec_lj_type", _ip), ("lig_lj_type", _ip),
        ("lig_ref_point", C.c_double * 3),
        ("n_swarms", C.c_int), ("n_glowworms", C.c_int),
    ]


class Tables(C.Structure):
    _fields_ = [("dfire_energy", _dp), ("lj_eps", _dp), ("lj_sigma", _dp)]


class GsoParams(C.Structure):
    _fields_ = [
        ("rho", C.c_double), ("gamma", C.c_double), ("beta", C.c_double),
        ("initial_luciferin", C.c_double), ("initial_vision_range", C.c_double),
        ("max_vision_range", C.c_double), ("max_neighbors", C.c_int),
        ("translation_step", C.c_double), ("rotation_step", C.c_double), ("nmodes_step", C.c_double),
    ]


class SwarmState(C.Structure):
    _fields_ = [
        ("pos", _dp), ("scoring", _dp), ("luciferin", _dp), ("vision_range", _dp),
        ("step", _ip), ("moved", _ip), ("nnei_len", _ip), ("select", _ip),
        ("ligand_reference_pose", _dp),
    ]


class Stats(C.Structure):
    _fields_ = [(n, C.c_longlong) for n in (
        "scored_poses", "steps", "pairs_fallback", "edge_d2_zero", "edge_d2_cutoff",
        "edge_u_zero", "edge_shortfall", "timeouts", "pairs_in_cutoff", "pairs_evaluated")]


class SynthSpec(C.Structure):
    _fields_ = [
        ("n_rec", C.c_int), ("n_lig", C.c_int), ("n_swarms", C.c_int), ("n_glowworms", C.c_int),
        ("n_modes_rec", C.c_int), ("n_modes_lig", C.c_int), ("seed", C.c_ulonglong),
    ]


# name -> (restype, argtypes) for every function declared in include/sparkle_b200.h
SIGNATURES = {
    "sd_last_error": (C.c_char_p, []),
    "sd_version": (C.c_char_p, []),
    "sd_device_count": (C.c_int, [_ip]),
    "sd_gso_params_default": (None, [C.POINTER(GsoParams)]),
    "sd_gso_draws": (C.c_int, [C.c_uint, C.c_int, C.c_int, C.c_int, _dp]),
    "sd_ctx_create": (C.c_int, [C.POINTER(ComplexDesc), C.c_int, C.POINTER(Tables), C.POINTER(GsoParams),
                                C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "sd_ctx_destroy": (C.c_int, [C.c_void_p]),
    "sd_ctx_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "sd_pose_len": (C.c_int, [C.c_void_p, C.c_int, _ip]),
    "sd_init_state": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "sd_set_state": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(SwarmState)]),
    "sd_get_state": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(SwarmState)]),
    "sd_set_draws": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int]),
    "sd_step": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "sd_get_stats": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "sd_get_tuning": (C.c_int, [C.c_void_p, _ip, _ip, _ip, _dp, C.c_int]),
    "sd_mixed_variant_count": (C.c_int, []),
    "sd_structure_load": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "sd_reference_point": (C.c_int, [_dp, C.c_int, _dp]),
    "sd_reference_point_device": (C.c_int, [C.c_int, _dp, C.c_int, _dp]),
    "sd_anm": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]),
    "sd_place_swarms": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_int, C.c_double, C.c_int, C.c_int, _dp, _dp]),
    "sd_cluster": (C.c_int, [C.c_void_p, C.c_int, _ip, _ip, _ip, _ip, _ip, _ip]),
    "sd_write_cluster_repr": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _dp]),
    "sd_starting_poses": (C.c_int, [_dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong, _dp]),
    "sd_structure_info": (C.c_int, [C.c_void_p, _ip, _ip]),
    "sd_structure_arrays": (C.c_int, [C.c_void_p, _dp, _ip, _ip, _ip, _dp]),
    "sd_structure_free": (C.c_int, [C.c_void_p]),
    "sd_write_pose_pdb": (C.c_int, [C.c_char_p, C.c_void_p, _dp, C.c_void_p, _dp]),
    "sd_write_checkpoint": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_longlong, C.c_longlong,
                                      C.POINTER(SwarmState)]),
    "sd_read_checkpoint": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_longlong),
                                     C.POINTER(C.c_longlong), C.POINTER(SwarmState)]),
    "sd_checkpoint_info": (C.c_int, [C.c_char_p, _ip, _ip, _ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "sd_materialise_poses": (C.c_int, [C.c_void_p, C.c_int, _ip, C.c_int, _dp, _dp]),
    "sd_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "sd_score_poses": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int, C.c_int, _dp, _dp]),
    "sd_score_poses_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_int]),
    "sd_dfire_bins": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int, _ip]),
    "sd_pydock_grad": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int, C.c_int, _dp, _dp]),
    "sd_write_gso_output": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _ip, _dp,
                                      _dp]),
    "sd_refine_poses": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int, C.c_int, C.c_double, C.c_int, _dp, _dp]),
    "sd_synth_buffer_size": (C.c_int, [C.POINTER(SynthSpec), C.POINTER(C.c_longlong)]),
    "sd_synth_generate": (C.c_int, [C.POINTER(SynthSpec), C.c_void_p, C.POINTER(ComplexDesc),
                                    C.POINTER(_dp)]),
    "sd_synth_tables": (C.c_int, [C.c_ulonglong, _dp, _dp, _dp]),
    "sd_crmath_eval": (C.c_int, [C.c_int, C.c_int, _dp, C.c_longlong, _dp]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libsparkle_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libsparkle_b200.so not built ({LIB_PATH}); run __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class SparkleError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib().sd_last_error().decode(errors="replace")
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


def check(code: int, where: str) -> None:
    if code != SD_OK:
        raise SparkleError(code, where)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)
