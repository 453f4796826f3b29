"""Luttinger-Tisza lower bound -- TEST INFRASTRUCTURE ONLY (oracle).

Restates src/luttinger_tisza.cpp with numpy: directed bonds from every one of
the 16 sublattices (build_bonds, :31-81; J1 XXZ as J1[I + (Delta-1) z_mu z_nu^T],
zero couplings skipped), M(k) = sum_bonds J e^{i k.d} in 3x3 blocks (:157-166),
the minimum eigenvalue over the L^3 k grid (:153-178), and E/spin = lambda_min/2
(:181). The reference's k vector is lattice_lib's wavevector_from_idx3; here
k = 2 pi K / (8 L) for the cubic supercell, the same grid as the SSF.
"""
from __future__ import annotations

import numpy as np

from . import System

LINK = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]])
FCC = np.array([[0, 0, 0], [0, 4, 4], [4, 0, 4], [4, 4, 0]])


def lt_minimum(L: int, J1: float, J2: float = 0.0, J3: float = 0.0, Delta: float = 1.0):
    """Returns (E_per_spin = lambda_min / 2, K_star) on the L^3 grid."""
    sys = System(1, J1=1.0, J2=1.0, J3=1.0, j1_mode=1)  # only for its displacement tables
    tables = {k: [sys.spec_displacements(spec, p) for p in range(4)] for k, spec in
              (("J1", 0), ("J2", 1), ("J3a", 2), ("J3b", 3))}
    r = np.array([LINK[s % 4] + FCC[s // 4] for s in range(16)])
    rmod = {tuple(x % 8): s for s, x in enumerate(r)}
    z = LINK / np.sqrt(3.0)
    bonds = []
    for name, j in (("J1", J1), ("J2", J2), ("J3a", J3), ("J3b", J3)):
        if j == 0.0:
            continue
        for a in range(16):
            for d in tables[name][a % 4]:
                b = rmod[tuple((r[a] + d) % 8)]
                if name == "J1" and Delta != 1.0:
                    M = j * (np.eye(3) + (Delta - 1.0) * np.outer(z[a % 4], z[b % 4]))
                else:
                    M = j * np.eye(3)
                bonds.append((a, b, np.array(d, float), M))
    best = (np.inf, None)
    for K0 in range(L):
        for K1 in range(L):
            for K2 in range(L):
                k = 2 * np.pi * np.array([K0, K1, K2]) / (8.0 * L)
                Mk = np.zeros((48, 48), complex)
                for a, b, d, M in bonds:
                    Mk[3 * a:3 * a + 3, 3 * b:3 * b + 3] += M * np.exp(1j * (k @ d))
                lmin = np.linalg.eigvalsh(Mk)[0]
                if lmin < best[0]:
                    best = (lmin, (K0, K1, K2))
    return 0.5 * best[0], best[1]
