"""Fitting couplings to a target static structure factor through the
differentiable energy and S(q).

spiral_byhand_spins(system, Q, replica)
    the spiral state of test/spiral_byhand.cpp:100-107: S_i = (0, cos q.x_i,
    sin q.x_i), q = 2 pi Q / (8L) for an integer index Q (lattice_lib's
    wavevector_from_idx3 of the L x L x L supercell).
zz_target(system, Q)
    S^zz(q) of that state, per k (the target of the gradient form's loss).
weighted_zz_loss(S, w, target)
    sum_q w(q) |S^zz(q) - S_target(q)|^2 per replica (S from autograd.ssf with
    "zz" among the correlators).
unrolled_quench(system, spins, params, steps, lr)
    projected gradient descent S <- normalise(S - lr (h - B)_tangent) for
    `steps` steps as a differentiable torch graph: the loss at the end can be
    differentiated with respect to the start spins and the couplings
    (autograd.LocalFieldFunction supplies the local field and its backward).
fit_couplings(system, spins0, target, w, params0, free, ...)
    Adam on the free entries of params = [J1, J2, J3, Bx, By, Bz] to make the
    quenched S^zz(q) of every replica match `target`.
"""
from __future__ import annotations

import numpy as np
import torch

from . import autograd as ag
from .engine import System


def spiral_byhand_spins(system: System, Q, replica: int = 0) -> np.ndarray:
    L = system.L[replica]
    pos, _ = system.positions(replica)
    q = 2 * np.pi * np.asarray(Q, dtype=np.float64) / (8 * L)
    ph = pos.astype(np.float64) @ q
    return np.stack([np.zeros_like(ph), np.cos(ph), np.sin(ph)], axis=1)


def zz_target(system: System, Q, zz_index: int = 0) -> np.ndarray:
    """S^zz(q) (real part) of the spiral state at index Q on a lattice of the
    system's size, computed by the system's own S(q) path (the correlators
    configured with ssf_configure; zz_index picks "zz"). Leaves replica 0's
    spins as they were."""
    keep = system.spins(0)
    system.set_spins(spiral_byhand_spins(system, Q, 0), 0)
    S = system.ssf_current(0)
    system.set_spins(keep, 0)
    return S[zz_index, :, 0].copy()


def weighted_zz_loss(S: torch.Tensor, w: torch.Tensor, target: torch.Tensor, zz_index: int = 0) -> torch.Tensor:
    """sum_q w(q) (Re S^zz(q) - target(q))^2 + w(q) (Im S^zz(q))^2 per
    replica: |S^zz - S_target|^2 with a real target."""
    d_re = S[:, zz_index, :, 0] - target
    d_im = S[:, zz_index, :, 1]
    return (w * (d_re ** 2 + d_im ** 2)).sum(dim=-1)


def unrolled_quench(system: System, spins: torch.Tensor, params: torch.Tensor | None, steps: int,
                    lr: float = 0.05) -> torch.Tensor:
    S = spins
    for _ in range(steps):
        h = ag.local_field(system, S, params)
        s3, h3 = S[:, :3], h[:, :3]
        t = h3 - (h3 * s3).sum(dim=1, keepdim=True) * s3
        n = s3 - lr * t
        n = n / n.norm(dim=1, keepdim=True)
        S = torch.cat([n, torch.zeros_like(S[:, 3:])], dim=1)
    return S


def fit_couplings(system: System, spins0: torch.Tensor, target: torch.Tensor, w: torch.Tensor,
                  params0, free=(1, 2), steps: int = 20, lr: float = 0.05, iters: int = 60,
                  step_size: float = 0.01, zz_index: int = 0):
    """Adam (step_size) on params[free] so that the S^zz(q) of every replica
    after `steps` quench steps from spins0 matches target; the loss is the
    weighted squared difference normalised by the target's weighted norm.
    Returns (params, loss history)."""
    p = torch.tensor(np.asarray(params0, dtype=np.float64), dtype=torch.float64, requires_grad=True)
    mask = torch.zeros(6, dtype=torch.float64)
    mask[list(free)] = 1.0
    opt = torch.optim.Adam([p], lr=step_size)
    norm = float((w * target ** 2).sum()) * system.R
    hist = []
    for _ in range(iters):
        opt.zero_grad()
        S = unrolled_quench(system, spins0, p, steps, lr)
        loss = weighted_zz_loss(ag.ssf(system, S), w, target, zz_index).sum() / norm
        loss.backward()
        p.grad *= mask
        opt.step()
        hist.append(float(loss.detach()))
    return p.detach().numpy(), np.array(hist)
