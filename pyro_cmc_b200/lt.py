"""Luttinger-Tisza bound on the GPU (src/luttinger_tisza.cpp, the ltgs program)
through pc_lt_minimum."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call


def lt_minimum(L: int, J1: float, J2: float = 0.0, J3: float = 0.0, Delta: float = 1.0):
    """Smallest eigenvalue of the 48 x 48 LT matrix over the L^3 grid
    k = 2 pi K / (8L). Returns dict(eigenvalue_map[L, L, L] (K order),
    E_min = lambda_min / 2 (energy per spin), k_star_idx[3], k_star_vec[3],
    eigenvector[48] complex (spin x, y, z of sublattice 0, 1, ...))."""
    n_k = L ** 3
    lam = np.empty(n_k)
    e = C.c_double(0.0)
    ks = np.zeros(3, dtype=np.int64)
    vec = np.empty((48, 2))
    call("pc_lt_minimum", int(L), float(J1), float(J2), float(J3), float(Delta),
         lam.ctypes.data_as(C.POINTER(C.c_double)), C.byref(e), ks.ctypes.data_as(C.POINTER(C.c_int64)),
         vec.ctypes.data_as(C.POINTER(C.c_double)))
    return dict(eigenvalue_map=lam.reshape(L, L, L), E_min=e.value, k_star_idx=ks,
                k_star_vec=2 * np.pi * ks / (8.0 * L), eigenvector=vec[:, 0] + 1j * vec[:, 1])
