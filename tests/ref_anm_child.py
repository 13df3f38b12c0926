"""Child process for the ANM pin: runs the reference's own cal_anm (compiled from its sources into
oracle/_ref/libsdref_anm.so, with its cuSOLVER eigensolver) on one PDB file and saves the modes and
re-centred coordinates.  A separate process because the reference's eigensolver ends with
cudaDeviceReset().  Usage: ref_anm_child.py pdb n_modes rmsd swarms glowworms out.npz"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pdb, n_modes, rmsd, swarms, glowworms, out = sys.argv[1], int(sys.argv[2]), float(sys.argv[3]), \
    int(sys.argv[4]), int(sys.argv[5]), sys.argv[6]
L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libsdref_anm.so"))
dp = C.POINTER(C.c_double)
L.ref_cal_anm.restype = C.c_int
L.ref_cal_anm.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, dp, dp,
                          C.c_int]
cap = 200000
modes = np.zeros(n_modes * cap * 3)
xyz = np.zeros(cap * 3)
n = L.ref_cal_anm(pdb.encode(), 1, 1, 1, n_modes, rmsd, swarms, glowworms, modes.ctypes.data_as(dp),
                  xyz.ctypes.data_as(dp), cap)
if n < 0:
    sys.exit(3)
np.savez(out, modes=modes[:n_modes * n * 3].reshape(n_modes, n, 3), xyz=xyz[:n * 3].reshape(n, 3))
