"""Helpers for the pyDock-style energy tests: oracle energy/gradient and finite differences
over translation, left tangent rotation (q <- exp(w/2) q) and ANM extents."""
import ctypes as C

import numpy as np

from oracle_bind import oracle

DP = C.POINTER(C.c_double)


def qmul(a, b):
    w1, x1, y1, z1 = a
    w2, x2, y2, z2 = b
    return np.array([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2])


def perturb(pose, k, h):
    """pose moved by h along gradient coordinate k (0-2 t, 3-5 rotation tangent, 6+ extents)."""
    p = np.array(pose, np.float64)
    if k < 3:
        p[k] += h
    elif k < 6:
        v = np.zeros(3)
        v[k - 3] = h
        dq = np.array([np.cos(h / 2), *(np.sin(h / 2) * v / h)])
        p[3:7] = qmul(dq, p[3:7])
    else:
        p[7 + (k - 6)] += h
    return p


def oracle_energy(osys, pose):
    pose = np.ascontiguousarray(pose, np.float64)
    return oracle().or_pydock_energy(osys.ptr, pose.ctypes.data_as(DP))


def oracle_grad(osys, pose, ng):
    pose = np.ascontiguousarray(pose, np.float64)
    g = np.zeros(ng)
    oracle().or_pydock_grad(osys.ptr, pose.ctypes.data_as(DP), g.ctypes.data_as(DP))
    return g


def fd_grad(osys, pose, ng, h=1e-4):
    return np.array([(oracle_energy(osys, perturb(pose, k, h)) - oracle_energy(osys, perturb(pose, k, -h))) / (2 * h)
                     for k in range(ng)])
