"""The differentiable form as the gradient configuration specifies it, through
the C ABI: a batch of uniform random configurations at L = 8 with
J = (1, 0.1, -0.05), B = (0.2, 0, 0); loss = sum_q w(q) |S^zz(q) - S_target(q)|^2
with w ~ U[0, 1] and S_target the S^zz(q) of the spiral_byhand state at a
seeded random Q (test/spiral_byhand.cpp:100-107); gradients with respect to
the spins (projected onto the tangent plane) and, through the energy, to
J1..J3 and B, against FP64 central differences (h = 1e-4) on the oracle.
Then the unrolled gradient quench (differentiable in the couplings) against
FP64 central differences of the same quench run on the oracle, and a fit of
(J2, J3) to a target S(q) that recovers the couplings that made it.

Tolerances: 2e-3 relative to the largest compared component (FP32 spins and
transforms against FP64), as the other finite-difference tests; the unrolled
quench (FP32 forward over several steps) 2e-2.
"""
import numpy as np
import pytest
import torch

import oracle
import pyro_cmc_b200 as pc
from pyro_cmc_b200 import autograd as ag
from pyro_cmc_b200 import ssf_fit

pytestmark = pytest.mark.gpu

C4 = dict(J1=1.0, J2=0.1, J3=-0.05, Delta=1.0, B=(0.2, 0.0, 0.0))
P4 = [1.0, 0.1, -0.05, 0.2, 0.0, 0.0]


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _oracle_objective(L, p, Ss, w, target, lam):
    """FP64: sum_r e_r + lam * sum_r sum_q w (S^zz_r - target)^2."""
    tot = 0.0
    for S in Ss:
        o = oracle.System(L, J1=p[0], J2=p[1], J3=p[2], B=p[3:6])
        o.set_spins(S)
        tot += o.energy()
        if lam:
            Z = o.ssf(["zz"], mode=2)[0]
            tot += lam * float((w * ((Z[:, 0] - target) ** 2 + Z[:, 1] ** 2)).sum())
    return tot


def test_config4_gradients_vs_central_differences():
    L, R = 8, 2
    rng = np.random.default_rng(4)
    g = pc.pyrochlore_system(L, n_replicas=R, seed=1, **C4)
    g.ssf_configure(["zz"], 0, [])
    Q = rng.integers(0, L, size=3)
    target = ssf_fit.zz_target(g, Q)
    assert target.max() > 1e5  # the spiral's Bragg peak
    for r in range(R):
        g.set_spins(_unit(rng, g.N(r)), r)
    w = rng.uniform(0, 1, L ** 3)
    lam = 1.0 / float((w * target ** 2).sum())
    Ss = [g.spins(r) for r in range(R)]
    spins = ag.spins_tensor(g).clone().requires_grad_(True)
    params = torch.tensor(P4, dtype=torch.float64, requires_grad=True)
    wt = torch.as_tensor(w, device="cuda")
    tt = torch.as_tensor(target, device="cuda")
    obj = ag.energy(g, spins, params).sum() + lam * ssf_fit.weighted_zz_loss(ag.ssf(g, spins), wt, tt).sum()
    obj.backward()
    gs = ag.project_tangent(spins.grad, spins.detach())[:, :3].cpu().numpy()
    gp = params.grad.numpy()
    h = 1e-4
    # couplings and field
    for k in range(6):
        dp = np.zeros(6)
        dp[k] = h
        fd = (_oracle_objective(L, np.array(P4) + dp, Ss, w, target, 0.0) -
              _oracle_objective(L, np.array(P4) - dp, Ss, w, target, 0.0)) / (2 * h)
        assert gp[k] == pytest.approx(fd, rel=2e-3, abs=2e-3 * max(1.0, abs(fd))), (k, gp[k], fd)
    # spins: tangent-projected gradients at a few sites of each replica
    got, ref = [], []
    for r in range(R):
        for i in rng.choice(g.N(r), size=6, replace=False):
            fd = np.zeros(3)
            for a in range(3):
                Sp = [S.copy() for S in Ss]
                Sm = [S.copy() for S in Ss]
                Sp[r][i, a] += h
                Sm[r][i, a] -= h
                fd[a] = (_oracle_objective(L, P4, [Sp[r]], w, target, lam) -
                         _oracle_objective(L, P4, [Sm[r]], w, target, lam)) / (2 * h)
            s = Ss[r][i]
            ref.append(fd - fd.dot(s) * s)
            got.append(gs[r * g.N(0) + i])
    got, ref = np.array(got), np.array(ref)
    assert np.abs(got - ref).max() <= 2e-3 * np.abs(ref).max(), (np.abs(got - ref).max(), np.abs(ref).max())


def _oracle_quench(L, p, S0, steps, lr):
    o = oracle.System(L, J1=p[0], J2=p[1], J3=p[2], B=p[3:6])
    S = S0.copy()
    for _ in range(steps):
        o.set_spins(S)
        hB = o.local_fields() - np.asarray(p[3:6])
        t = hB - (hB * S).sum(1, keepdims=True) * S
        S = S - lr * t
        S /= np.linalg.norm(S, axis=1, keepdims=True)
    o.set_spins(S)
    return o.ssf(["zz"], mode=2)[0]


def test_unrolled_quench_coupling_gradient_vs_central_differences():
    L, R, steps, lr = 3, 2, 6, 0.05
    rng = np.random.default_rng(9)
    g = pc.pyrochlore_system(L, n_replicas=R, seed=2, **C4)
    g.ssf_configure(["zz"], 0, [])
    S0 = [_unit(rng, g.N(r)) for r in range(R)]
    for r in range(R):
        g.set_spins(S0[r], r)
    w = rng.uniform(0, 1, L ** 3)
    target = ssf_fit.zz_target(g, rng.integers(0, L, size=3))
    for r in range(R):
        g.set_spins(S0[r], r)
    spins0 = ag.spins_tensor(g).clone()
    params = torch.tensor(P4, dtype=torch.float64, requires_grad=True)
    S = ssf_fit.unrolled_quench(g, spins0, params, steps, lr)
    loss = ssf_fit.weighted_zz_loss(ag.ssf(g, S), torch.as_tensor(w, device="cuda"),
                                    torch.as_tensor(target, device="cuda")).sum()
    loss.backward()
    S32 = [spins0[r * g.N(0):(r + 1) * g.N(0), :3].cpu().numpy().astype(np.float64) for r in range(R)]

    def f(p):
        tot = 0.0
        for r in range(R):
            Z = _oracle_quench(L, p, S32[r], steps, lr)
            tot += float((w * ((Z[:, 0] - target) ** 2 + Z[:, 1] ** 2)).sum())
        return tot

    h = 1e-4
    fd = []
    for k in range(6):
        dp = np.zeros(6)
        dp[k] = h
        fd.append((f(np.array(P4) + dp) - f(np.array(P4) - dp)) / (2 * h))
    fd = np.array(fd)
    got = params.grad.numpy()
    assert np.abs(got - fd).max() <= 2e-2 * np.abs(fd).max(), (got, fd)


def test_fit_recovers_couplings_from_quenched_ssf():
    """Target: S^zz(q) after a 20-step quench from fixed random starts with
    J = (1, 0.1, -0.05), B = (0.2, 0, 0). Fit (J2, J3) from (0, 0) through the
    unrolled quench; the fit lands within 0.01 of the true couplings."""
    L, R, steps, lr = 4, 4, 20, 0.05
    rng = np.random.default_rng(21)
    g = pc.pyrochlore_system(L, n_replicas=R, seed=3, **C4)
    g.ssf_configure(["zz"], 0, [])
    for r in range(R):
        g.set_spins(_unit(rng, g.N(r)), r)
    spins0 = ag.spins_tensor(g).clone()
    true = torch.tensor(P4, dtype=torch.float64)
    with torch.no_grad():
        S_t = ssf_fit.unrolled_quench(g, spins0, true, steps, lr)
        target_r = ag.ssf(g, S_t)[:, 0, :, 0]  # per replica
    w = torch.ones(L ** 3, dtype=torch.float64, device="cuda")
    # one target per replica: broadcast through the loss
    p, hist = ssf_fit.fit_couplings(g, spins0, target_r, w, [1.0, 0.0, 0.0, 0.2, 0.0, 0.0], free=(1, 2),
                                    steps=steps, lr=lr, iters=80, step_size=0.01)
    assert hist[-1] < 1e-2 * hist[0], hist[[0, -1]]
    assert abs(p[1] - 0.1) < 0.01 and abs(p[2] + 0.05) < 0.01, p


def test_device_output_energy_and_gradient_match_the_host_calls():
    """pc_energy_device and pc_energy_grad_device (results left on the device,
    queued without waiting) give the host calls' energies, spin gradient and
    per-replica sums bit for bit, with and without the coupling products, with
    the upstream g on the device or 1 for every replica."""
    import torch

    s = pc.pyrochlore_system([4, 4, 4], J1=1.0, J2=0.1, J3=-0.05, B=(0.2, 0.0, 0.1), seed=2)
    s.random_spins(9)
    R, ns = s.R, len(s.spec_names)
    nc = np.array([s.Nc(r) for r in range(R)], dtype=np.float64)
    e_host, _ = s.energy()
    e_dev = torch.empty(R, dtype=torch.float64, device="cuda")
    s.energy_device(e_dev.data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(e_dev.cpu().numpy(), e_host)
    up = np.array([0.5, -1.0, 2.0])
    for couplings in (True, False):
        gs_host = torch.empty((s.N_total, 4), dtype=torch.float32, device="cuda")
        e2, gJ, gB = s.energy_grad(up, gs_host.data_ptr(), couplings=couplings)
        gs = torch.empty_like(gs_host)
        sums = torch.zeros((R, 4 + 9 * ns), dtype=torch.float64, device="cuda")
        gd = torch.as_tensor(up, device="cuda")
        s.energy_grad_device(gd.data_ptr(), gs.data_ptr(), sums.data_ptr(), couplings)
        torch.cuda.synchronize()
        assert torch.equal(gs, gs_host)
        v = sums.cpu().numpy()
        np.testing.assert_array_equal(v[:, 0] / nc, e2)
        np.testing.assert_array_equal(-up[:, None] * v[:, 1:4] / nc[:, None], gB)
        if couplings:
            np.testing.assert_array_equal(up[:, None] * v[:, 4:] / nc[:, None], gJ.reshape(R, -1))
        else:
            assert (v[:, 4:] == 0).all()
    sums = torch.zeros((R, 4 + 9 * ns), dtype=torch.float64, device="cuda")
    s.energy_grad_device(None, None, sums.data_ptr(), False)
    torch.cuda.synchronize()
    e3, _, gB3 = s.energy_grad(None, None, couplings=False)
    v = sums.cpu().numpy()
    np.testing.assert_array_equal(v[:, 0] / nc, e3)
    np.testing.assert_array_equal(-v[:, 1:4] / nc[:, None], gB3)


def test_kept_ssf_amplitudes_give_the_recomputed_backward():
    """pc_ssf_forward_keep / pc_ssf_backward_kept: the forward values equal
    pc_ssf_forward's, and the backward from the kept amplitudes equals
    pc_ssf_backward's (which recomputes the transform) bit for bit; a token
    made stale by a later forward on other spins falls back to recomputing."""
    s = pc.pyrochlore_system([4, 4, 6], J1=1.0, J2=0.1, seed=3)
    s.ssf_configure(["zz", "xy"], 0, [])
    s.random_spins(4)
    A = ag.spins_tensor(s).clone()
    out = torch.empty((s.R, s.n_corr, s.Nc(0), 2), dtype=torch.float64, device="cuda")
    n_val = sum(s.n_corr * s.Nc(r) * 2 for r in range(s.R))
    out = torch.empty(n_val, dtype=torch.float64, device="cuda")
    go = torch.randn(n_val, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    ref = torch.empty((s.N_total, 4), dtype=torch.float32, device="cuda")
    s.ssf_backward_device(go.data_ptr(), ref.data_ptr())
    ref_val = torch.empty_like(out)
    s.ssf_forward_device(ref_val.data_ptr())
    t1 = s.ssf_forward_keep(out.data_ptr())
    torch.cuda.synchronize()
    assert t1 != 0 and torch.equal(out, ref_val)
    got = torch.empty_like(ref)
    s.ssf_backward_kept(t1, go.data_ptr(), got.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(got, ref)
    # stale: a forward on other spins in between, then the first spins again
    t1 = s.ssf_forward_keep(out.data_ptr())
    s.random_spins(5)
    t2 = s.ssf_forward_keep(out.data_ptr())
    torch.cuda.synchronize()
    assert t2 != t1
    ag.spins_tensor(s).copy_(A)
    torch.cuda.synchronize()
    got = torch.empty_like(ref)
    s.ssf_backward_kept(t1, go.data_ptr(), got.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(got, ref)


@pytest.mark.parametrize("J2", [0.1, 0.0])
def test_isotropic_parameter_gradient_from_the_energy_pass(J2):
    """With isotropic J1, J2, J3 (Delta = 1, every group nonzero) the gradient
    in [J1, J2, J3, B] comes from the forward energy pass's per-group bond sums
    (pc_energy_groups_device); it agrees with the general path's coupling
    products (pc_energy_grad) to the rounding of the FP32 per-cell sums. With
    J2 = 0 (its group skipped by the energy pass) the general path runs."""
    s = pc.pyrochlore_system(6, n_replicas=4, J1=1.0, J2=J2, J3=-0.05, B=(0.2, 0.0, 0.1), seed=8)
    s.random_spins(12)
    spins = ag.spins_tensor(s).clone().requires_grad_(True)
    params = torch.tensor([1.0, J2, -0.05, 0.2, 0.0, 0.1], dtype=torch.float64, requires_grad=True)
    up = torch.tensor([0.3, -1.0, 2.0, 0.5], dtype=torch.float64, device="cuda")
    e = ag.energy(s, spins, params)
    (e * up).sum().backward()
    gs_ref = torch.empty_like(spins)
    e2, gJ, gB = s.energy_grad(up.cpu().numpy(), gs_ref.data_ptr(), couplings=True)
    ref = ag._param_grads(s, gJ, gB).sum(axis=0)
    np.testing.assert_allclose(params.grad.numpy(), ref, rtol=1e-5, atol=1e-7 * np.abs(ref).max())
    np.testing.assert_allclose(e.detach().cpu().numpy(), e2, rtol=1e-5)
    torch.testing.assert_close(spins.grad, gs_ref, rtol=1e-5, atol=1e-6)
