"""Differentiable energy and S(q) as torch.autograd.Functions over the C ABI.

Spins are a float32 CUDA tensor [N_total, 4] (x, y, z, unused) in the
engine's layout: replicas back to back, each sublattice-major
(site = sl*Nc + cell). Energies are per cubic cell, float64 [R]. S(q) is
float64 [R, n_corr, n_k, 2] (Re, Im) for the correlators configured with
System.ssf_configure.

  energy(system, spins, params=None) -> e[R]
      d/dspins: g/Nc * (h_i - B) (the reference's local field minus the
      global field, src/MC.cpp:113); d/dparams for params = [J1, J2, J3, Bx,
      By, Bz] of a pyrochlore system (define_pyrochlore): dE/dJ1 sums the six
      pair specs through J1[I + (Delta-1) z_mu z_nu], dE/dJ3 the J3a and J3b
      specs. Hand-written kernel (pc_energy_grad).
  ssf(system, spins) -> S
      backward recomputes the forward transform and applies its adjoint
      (pc_ssf_backward); no transform is stored.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import ERR_UNSUPPORTED, PyroCMCError
from .engine import PAIRS, System, local_axis


class _DeviceArray:
    """Exposes a raw device pointer to torch through __cuda_array_interface__."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": tuple(shape), "typestr": typestr,
                                         "version": 3, "strides": None}


def spins_tensor(system: System) -> torch.Tensor:
    """The system's own device spin buffer as a [N_total, 4] float32 tensor
    (a view, no copy)."""
    ptr = system.spins_device_ptr(0)
    view = getattr(system, "_spins_view", None)
    if view is None or view[0] != ptr:
        view = (ptr, torch.as_tensor(_DeviceArray(ptr, (system.N_total, 4), "<f4"), device="cuda"))
        system._spins_view = view
    return view[1].detach()  # a new tensor object on the same memory each call


def _order(system: System):
    """Orders the system's next calls after the work queued on the current
    torch stream: nothing to do when the system runs on that stream
    (System.set_stream), else the host waits for the stream."""
    if getattr(system, "stream_ptr", None) != torch.cuda.current_stream().cuda_stream:
        torch.cuda.current_stream().synchronize()


def _join(system: System):
    """Orders the current torch stream after the system's queued work (the
    device-output calls return without waiting)."""
    if getattr(system, "stream_ptr", None) != torch.cuda.current_stream().cuda_stream:
        torch.cuda.synchronize()


def _load(system: System, spins: torch.Tensor):
    if spins.shape != (system.N_total, 4) or spins.dtype != torch.float32 or not spins.is_cuda:
        raise ValueError("spins must be a float32 CUDA tensor of shape [N_total, 4]")
    dst = spins_tensor(system)
    if spins.data_ptr() != dst.data_ptr():
        dst.copy_(spins.detach())
        _order(system)


def _apply_params(system: System, params: torch.Tensor):
    """Sets J1, J2, J3 and B of a pyrochlore system from params[6]."""
    pp = getattr(system, "pyro_params", None)
    if pp is None:
        raise ValueError("params need a system built with define_pyrochlore")
    J1, J2, J3, bx, by, bz = [float(x) for x in params.detach().cpu().tolist()]
    if (J1, J2, J3) != (pp["J1"], pp["J2"], pp["J3"]):
        I3 = np.eye(3)
        mats = []
        if pp["split_J1"]:
            for mu, nu in PAIRS:
                mats.append(J1 * (I3 + (pp["Delta"] - 1.0) * np.outer(local_axis(mu), local_axis(nu))))
        else:
            mats.append(J1 * I3)
        mats += [J2 * I3, J3 * I3, J3 * I3]
        system.set_coupling_matrices(range(len(mats)), mats)  # one rebuild of the tables
        pp.update(J1=J1, J2=J2, J3=J3)
    system.set_global_field([bx, by, bz])


def _param_grads(system: System, gJ: np.ndarray, gB: np.ndarray) -> np.ndarray:
    """dE/d[J1, J2, J3, Bx, By, Bz] per replica from the per-spec matrix grads."""
    pp = system.pyro_params
    R = gJ.shape[0]
    out = np.zeros((R, 6))
    k = 0
    I3 = np.eye(3)
    if pp["split_J1"]:
        for mu, nu in PAIRS:
            dM = I3 + (pp["Delta"] - 1.0) * np.outer(local_axis(mu), local_axis(nu))
            out[:, 0] += np.einsum("rab,ab->r", gJ[:, k], dM)
            k += 1
    else:
        out[:, 0] += np.einsum("raa->r", gJ[:, k])
        k += 1
    out[:, 1] = np.einsum("raa->r", gJ[:, k])
    out[:, 2] = np.einsum("raa->r", gJ[:, k + 1]) + np.einsum("raa->r", gJ[:, k + 2])
    out[:, 3:] = gB
    return out


def _param_grads_device(system: System, gJ: torch.Tensor, gB: torch.Tensor) -> torch.Tensor:
    """_param_grads on device tensors: gJ [R, n_spec, 3, 3], gB [R, 3] -> [R, 6]."""
    key = (gJ.device, gJ.shape[1])
    cache = getattr(system, "_dparam_mats", None)
    if cache is None or cache[0] != key:
        # d(spec matrix)/dJ1, dJ2, dJ3 per spec
        pp = system.pyro_params
        D = np.zeros((3, gJ.shape[1], 3, 3))
        k = 0
        I3 = np.eye(3)
        if pp["split_J1"]:
            for mu, nu in PAIRS:
                D[0, k] = I3 + (pp["Delta"] - 1.0) * np.outer(local_axis(mu), local_axis(nu))
                k += 1
        else:
            D[0, k] = I3
            k += 1
        D[1, k] = I3
        D[2, k + 1] = I3
        D[2, k + 2] = I3
        cache = (key, torch.as_tensor(D, dtype=torch.float64, device=gJ.device))
        system._dparam_mats = cache
    return torch.cat([torch.einsum("rsab,jsab->rj", gJ, cache[1]), gB], dim=1)


class EnergyFunction(torch.autograd.Function):
    """e_per_cell[r] of every replica (total_energy_per_unit_cell,
    src/MC.cpp:305-312) with its gradients in the spins and, given params
    [J1, J2, J3, Bx, By, Bz], in those; results stay on the device (the
    device-output entry points, ordered by stream)."""

    @staticmethod
    def forward(ctx, spins, params, system):
        if params is not None:
            _apply_params(system, params)
        _load(system, spins)
        e = torch.empty(system.R, dtype=torch.float64, device=spins.device)
        ctx.groups = None
        if params is not None and system.pyro_params["Delta"] == 1.0:
            # isotropic J1, J2, J3: dE/dJ are the groups' bare bond sums, which
            # the energy pass forms anyway (pc_energy_groups_device)
            groups = torch.empty((system.R, 9), dtype=torch.float64, device=spins.device)
            try:
                system.energy_groups_device(e.data_ptr(), groups.data_ptr())
                ctx.groups = groups
            except PyroCMCError as err:
                if err.code != ERR_UNSUPPORTED:
                    raise
        if ctx.groups is None:
            system.energy_device(e.data_ptr())
        _join(system)
        ctx.system = system
        ctx.has_params = params is not None
        ctx.params_device = params.device if params is not None else None
        ctx.save_for_backward(spins)
        return e

    @staticmethod
    def backward(ctx, grad_e):
        system = ctx.system
        (spins,) = ctx.saved_tensors
        _load(system, spins)
        g = grad_e.detach().to(device=spins.device, dtype=torch.float64).contiguous()
        grad_spins = torch.empty_like(spins)  # every site is written
        n_spec = len(system.spec_names)
        sums = torch.zeros((system.R, 4 + 9 * n_spec), dtype=torch.float64, device=spins.device)
        _order(system)
        fast = ctx.groups is not None
        system.energy_grad_device(g.data_ptr(), grad_spins.data_ptr(), sums.data_ptr(),
                                  couplings=ctx.has_params and not fast)
        _join(system)
        gp = None
        if fast:
            s = g / torch.as_tensor(_nc_vector(system), device=spins.device)
            G = ctx.groups
            dj = torch.stack([G[:, 0] + G[:, 1] + G[:, 2], G[:, 3], G[:, 4] + G[:, 5]], dim=1)
            gp = torch.cat([s[:, None] * dj, -s[:, None] * G[:, 6:9]], dim=1).sum(dim=0).to(ctx.params_device)
        elif ctx.has_params:
            s = g / torch.as_tensor(_nc_vector(system), device=spins.device)
            gJ = (s[:, None] * sums[:, 4:]).reshape(system.R, n_spec, 3, 3)
            gB = -s[:, None] * sums[:, 1:4]
            gp = _param_grads_device(system, gJ, gB).sum(dim=0).to(ctx.params_device)
        return grad_spins, gp, None


class SSFFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, spins, system):
        _load(system, spins)
        nk = system.Nc(0)
        out = torch.empty((system.R, system.n_corr, nk, 2), dtype=torch.float64, device=spins.device)
        _order(system)
        ctx.token = system.ssf_forward_keep(out.data_ptr())  # the amplitudes stay for the backward
        _join(system)
        ctx.system = system
        ctx.save_for_backward(spins)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        system = ctx.system
        (spins,) = ctx.saved_tensors
        _load(system, spins)
        go = grad_out.detach().to(torch.float64).contiguous()
        grad_spins = torch.empty_like(spins)
        _order(system)
        system.ssf_backward_kept(ctx.token, go.data_ptr(), grad_spins.data_ptr())
        _join(system)
        return grad_spins, None


def _nc_vector(system: System) -> np.ndarray:
    return np.array([system.Nc(r) for r in range(system.R)], dtype=np.float64)


def _field_of(system: System, field: torch.Tensor, couplings: bool):
    """h(field) - B per site (float32 [N_total, 4], fourth component 0) and,
    with couplings, the per-replica bond sums P(field)[spec] = sum over the
    spec's bonds of field_src field_tgt^T (pc_energy_grad_field with g = Nc)."""
    field = field.detach().contiguous()
    out = torch.empty_like(field)
    _order(system)
    _, P, _ = system.energy_grad_field(field.data_ptr(), _nc_vector(system), out.data_ptr(), couplings=couplings)
    return out, P


class LocalFieldFunction(torch.autograd.Function):
    """h_i(S; J) - B for every site (MC_runner::local_field minus the global
    field, src/MC.cpp:87-96,113): the energy's spin gradient times Nc. Its
    backward is exact for the bilinear energy: with upstream u,
    d(sum u.h)/dS = h(u) (the coupling matrix is the Hessian), d/dJ_spec =
    sum over the spec's bonds of u_src S_tgt^T + S_src u_tgt^T (formed from
    the bond sums as P(S + a u) - P(S) - P(a u), divided by a, with a scaling
    u to the spins' magnitude), d/dB = -sum_i u_i."""

    @staticmethod
    def forward(ctx, spins, params, system):
        if params is not None:
            _apply_params(system, params)
        h, _ = _field_of(system, spins, couplings=False)
        ctx.system = system
        ctx.has_params = params is not None
        ctx.params_device = params.device if params is not None else None
        ctx.save_for_backward(spins)
        return h

    @staticmethod
    def backward(ctx, grad_h):
        system = ctx.system
        (spins,) = ctx.saved_tensors
        u = grad_h.detach().clone()
        u[:, 3] = 0
        B = torch.as_tensor(system.get_global_field(), dtype=torch.float32, device=u.device)
        hu, _ = _field_of(system, u, couplings=False)
        grad_spins = hu
        grad_spins[:, :3] += B  # h(u), without the field
        gp = None
        if ctx.has_params:
            s = spins.detach().clone()
            s[:, 3] = 0
            a = float(s[:, :3].norm()) / max(float(u[:, :3].norm()), 1e-30)
            _, P_sum = _field_of(system, s + a * u, couplings=True)
            _, P_s = _field_of(system, s, couplings=True)
            _, P_u = _field_of(system, a * u, couplings=True)
            mixed = (P_sum - P_s - P_u) / a  # [R, spec, 3, 3]
            R = system.R
            gB = np.zeros((R, 3))
            off = 0
            for r in range(R):
                n = system.N(r)
                gB[r] = -u[off:off + n, :3].sum(dim=0).double().cpu().numpy()
                off += n
            gp = torch.as_tensor(_param_grads(system, mixed, gB).sum(axis=0), dtype=torch.float64,
                                 device=ctx.params_device)
        return grad_spins, gp, None


def local_field(system: System, spins: torch.Tensor, params: torch.Tensor | None = None) -> torch.Tensor:
    """h_i - B of every site, differentiable in the spins and params."""
    return LocalFieldFunction.apply(spins, params, system)


def energy(system: System, spins: torch.Tensor, params: torch.Tensor | None = None) -> torch.Tensor:
    return EnergyFunction.apply(spins, params, system)


def ssf(system: System, spins: torch.Tensor) -> torch.Tensor:
    if len(set(system.L)) != 1:
        raise ValueError("the differentiable S(q) needs replicas of one size")
    return SSFFunction.apply(spins, system)


def project_tangent(grad: torch.Tensor, spins: torch.Tensor) -> torch.Tensor:
    """Removes the radial part of a spin gradient: g - (g.S) S (spins stay on S^2)."""
    S = spins[:, :3]
    g = grad[:, :3]
    out = torch.zeros_like(grad)
    out[:, :3] = g - (g * S).sum(dim=1, keepdim=True) * S
    return out


def gradient_quench(system: System, steps: int = 500, lr: float = 0.05) -> np.ndarray:
    """Projected gradient descent of the energy on S^2 for every replica
    (S <- normalise(S - lr * tangent grad)), from the system's current spins.
    Returns the energy per cubic cell of each replica after every step."""
    spins = spins_tensor(system)
    hist = []
    for _ in range(steps):
        g = torch.empty_like(spins)  # every site is written
        e, _, _ = system.energy_grad(None, g.data_ptr(), couplings=False)
        hist.append(e)
        t = project_tangent(g, spins)
        new = spins[:, :3] - lr * t[:, :3]
        new = new / new.norm(dim=1, keepdim=True)
        spins[:, :3] = new
        _order(system)
    e, _ = system.energy()
    hist.append(e)
    return np.array(hist)
