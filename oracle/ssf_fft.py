"""Test infrastructure: the static structure factor of ssf_manager::sample
(include/ssf_manager.hpp:260-293) restated with numpy FFTs, for lattices too
large for the oracle's O(N n_k) direct sum. Only the tests and the bench's
checker import this module.

Per spin component a and sublattice sl, A^a_sl(K) is the 3-D DFT over cells
(forward sign, unnormalised) of S^a on that sublattice; the reference contracts
sum_{mu nu} exp(+i q.(r_mu - r_nu)) conj(A^a_mu) A^b_nu, which equals
conj(B^a) B^b with B^a(K) = sum_sl exp(-i q.r_sl) A^a_sl(K), q = 2 pi K/(8L).
Flat k in C order over (K0, K1, K2) = (Kx, Ky, Kz); cell = cx + L(cy + L cz).
Sublattice offsets r_sl = link[p] + R_fcc[f], sl = 4f + p
(include/pyrochlore_geometry.hpp:16-29).
"""
from __future__ import annotations

import numpy as np

LINK = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]])
R_FCC = np.array([[0, 0, 0], [0, 4, 4], [4, 0, 4], [4, 4, 0]])
R_SL = np.array([LINK[sl % 4] + R_FCC[sl // 4] for sl in range(16)])
AXIS = {"x": 0, "y": 1, "z": 2}


def amplitudes(S: np.ndarray, L: int) -> np.ndarray:
    """B^a(k) for spins S[16*L^3, 3] in storage order; returns complex [3, L^3]."""
    S = np.asarray(S, dtype=np.float64).reshape(16, L, L, L, 3)  # [sl][cz][cy][cx][a]
    K = np.arange(L)
    B = np.zeros((3, L, L, L), dtype=np.complex128)  # [a][Kx][Ky][Kz]
    for sl in range(16):
        F = np.fft.fftn(S[sl], axes=(0, 1, 2))  # [Kz][Ky][Kx][a]
        F = np.transpose(F, (3, 2, 1, 0))  # [a][Kx][Ky][Kz]
        r = R_SL[sl]
        ph = [np.exp(-2j * np.pi * K * r[d] / (8 * L)) for d in range(3)]
        B += F * ph[0][:, None, None] * ph[1][None, :, None] * ph[2][None, None, :]
    return B.reshape(3, L ** 3)


def sublattice_ft(S: np.ndarray, L: int) -> np.ndarray:
    """save_ft_spin_state's spin_ft (src/MC.cpp:320-368): per component a and
    sublattice sl the 3-D DFT over cells (forward sign, unnormalised) of S^a
    on that sublattice, without the sublattice phase. Returns complex
    [3, 16, L^3], k flat in C order over (Kx, Ky, Kz)."""
    S = np.asarray(S, dtype=np.float64).reshape(16, L, L, L, 3)  # [sl][cz][cy][cx][a]
    F = np.fft.fftn(S, axes=(1, 2, 3))  # [sl][Kz][Ky][Kx][a]
    return np.transpose(F, (4, 0, 3, 2, 1)).reshape(3, 16, L ** 3)


def ssf(S: np.ndarray, L: int, corr) -> np.ndarray:
    """S^{ab}(k) = conj(B^a) B^b for each correlator name; [n_corr, L^3, 2]."""
    B = amplitudes(S, L)
    out = np.empty((len(corr), L ** 3, 2))
    for c, name in enumerate(corr):
        v = np.conj(B[AXIS[name[0]]]) * B[AXIS[name[1]]]
        out[c, :, 0] = v.real
        out[c, :, 1] = v.imag
    return out


def adjoint(S: np.ndarray, L: int, corr, dval: np.ndarray) -> np.ndarray:
    """dLoss/dS_i^c for dLoss/dS^{ab}(k) = dval[n_corr, L^3, 2] (real, imag
    parts): Re sum_k exp(+i q.x_i) Y^c(k), Y^c = sum over correlators of
    [c == a] conj(D) B^b + [c == b] D B^a, D = dval[..., 0] + i dval[..., 1].
    Returns [16*L^3, 3] in storage order."""
    B = amplitudes(S, L)
    Y = np.zeros_like(B)
    for c, name in enumerate(corr):
        a, b = AXIS[name[0]], AXIS[name[1]]
        D = dval[c, :, 0] + 1j * dval[c, :, 1]
        Y[a] += np.conj(D) * B[b]
        Y[b] += D * B[a]
    Y = Y.reshape(3, L, L, L)  # [a][Kx][Ky][Kz]
    K = np.arange(L)
    out = np.empty((16, L, L, L, 3))  # [sl][cz][cy][cx][a]
    for sl in range(16):
        r = R_SL[sl]
        ph = [np.exp(+2j * np.pi * K * r[d] / (8 * L)) for d in range(3)]
        Z = Y * ph[0][None, :, None, None] * ph[1][None, None, :, None] * ph[2][None, None, None, :]
        G = np.fft.ifftn(Z, axes=(1, 2, 3)) * L ** 3  # [a][cx][cy][cz], exp(+)
        out[sl] = np.transpose(G.real, (3, 2, 1, 0))
    return out.reshape(16 * L ** 3, 3)
