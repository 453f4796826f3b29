"""CUDA path (through the C ABI): energy / S(q) gradients against FP64 finite
differences on the oracle, batched parallel tempering, and statistical parity
of annealing and tempering with the reference-faithful oracle.

Tolerances: gradients 1e-5 relative to the largest component against the
oracle's analytic gradients; against FP64 central differences (h = 1e-4),
2e-3 relative (FP32 transforms on the GPU side). Stochastic observables: per
temperature |difference| within 3 sigma of the combined standard error, with
at least 95% of temperatures inside and none beyond 5 sigma (many
temperatures are tested at once).
"""
import concurrent.futures as cf

import numpy as np
import pytest
import torch

import oracle
import oracle.lt
import pyro_cmc_b200 as pc
from pyro_cmc_b200 import autograd as ag

pytestmark = pytest.mark.gpu

C4 = dict(J1=1.0, J2=0.1, J3=-0.05, Delta=1.0, B=(0.2, 0.0, 0.0))


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def test_energy_grad_matches_oracle():
    c = dict(J1=1.0, J2=0.1, J3=-0.05, Delta=0.6, B=(0.2, -0.1, 0.3))
    L = 3
    g = pc.pyrochlore_system(L, **c)
    o = oracle.System(L, **c)
    rng = np.random.default_rng(0)
    g.set_spins(unit(rng, g.N()))
    S = g.spins()
    o.set_spins(S)
    grad = torch.zeros((g.N_total, 4), dtype=torch.float32, device="cuda")
    e, gJ, gB = g.energy_grad(None, grad.data_ptr())
    Nc = L ** 3
    assert e[0] == pytest.approx(o.energy(), abs=1e-5 * 100)
    ref_gs = (o.local_fields() - np.array(c["B"])) / Nc
    gs = grad[:, :3].cpu().numpy()
    assert np.abs(gs - ref_gs).max() <= 1e-5 * np.abs(ref_gs).max()
    ref_gJ = o.coupling_grads() / Nc
    assert np.abs(gJ[0] - ref_gJ).max() <= 1e-5 * max(1.0, np.abs(ref_gJ).max())
    np.testing.assert_allclose(gB[0], -S.sum(axis=0) / Nc, atol=1e-6 * g.N())


@pytest.mark.parametrize("L,R,threads", [(3, 1, 128), (8, 3, 128), (8, 2, 64), (12, 1, 256)])
def test_structured_energy_grad_matches_generic_and_oracle(L, R, threads):
    """The structured gradient kernel (work items of up to two tiles per
    thread, per-warp rows) against the generic bond-table kernel and, for
    replica 0, the oracle; without coupling gradients it gives the same energy,
    spin gradient and field gradient."""
    c = dict(J1=1.0, J2=0.1, J3=-0.05, Delta=0.6, B=(0.2, -0.1, 0.3))
    g = pc.pyrochlore_system(L, n_replicas=R, **c)
    g.set_tile(threads, 4)
    rng = np.random.default_rng(L + R)
    for r in range(R):
        g.set_spins(unit(rng, g.N(r)), r)
    up = np.linspace(1.0, -0.5, R)
    res = {}
    for generic in (False, True):
        g.set_kernel_path(generic)
        grad = torch.zeros((g.N_total, 4), dtype=torch.float32, device="cuda")
        e, gJ, gB = g.energy_grad(up, grad.data_ptr())
        res[generic] = (e, gJ, gB, grad.cpu().numpy())
    g.set_kernel_path(False)
    grad = torch.full((g.N_total, 4), 7.0, dtype=torch.float32, device="cuda")
    e2, gJ2, gB2 = g.energy_grad(up, grad.data_ptr(), couplings=False)
    assert gJ2 is None
    (e, gJ, gB, gs), (eg, gJg, gBg, gsg) = res[False], res[True]
    np.testing.assert_allclose(e, eg, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(gB, gBg, rtol=1e-6, atol=1e-6)
    assert np.abs(gs - gsg).max() <= 1e-5 * np.abs(gsg).max()
    assert np.abs(gJ - gJg).max() <= 1e-5 * max(1.0, np.abs(gJg).max())
    np.testing.assert_allclose(e2, e, rtol=1e-6, atol=1e-6)
    np.testing.assert_array_equal(gB2, gB)
    g2 = grad.cpu().numpy()
    assert np.abs(g2 - gs).max() <= 1e-5 * np.abs(gs).max()  # every site written
    assert np.all(g2[:, 3] == 0)
    o = oracle.System(L, **c)
    o.set_spins(g.spins(0))
    Nc = L ** 3
    ref_gJ = up[0] * o.coupling_grads() / Nc
    assert np.abs(gJ[0] - ref_gJ).max() <= 1e-5 * max(1.0, np.abs(ref_gJ).max())
    assert e[0] == pytest.approx(o.energy(), abs=1e-5 * 100)


def test_energy_autograd_params_vs_finite_differences():
    L = 2
    g = pc.pyrochlore_system(L, n_replicas=2, **C4)
    rng = np.random.default_rng(1)
    S0 = unit(rng, g.N())
    S1 = unit(rng, g.N())
    g.set_spins(S0, 0)
    g.set_spins(S1, 1)
    spins = ag.spins_tensor(g).clone().requires_grad_(True)
    params = torch.tensor([1.0, 0.1, -0.05, 0.2, 0.0, 0.0], dtype=torch.float64, requires_grad=True)
    e = ag.energy(g, spins, params)
    w = torch.tensor([1.0, -0.5], dtype=torch.float64, device="cuda")
    (e * w).sum().backward()
    # FP64 central differences on the oracle, h = 1e-4
    h = 1e-4
    Ss = [g.spins(0), g.spins(1)]

    def loss(p):
        tot = 0.0
        for r, wr in enumerate([1.0, -0.5]):
            o = oracle.System(L, J1=p[0], J2=p[1], J3=p[2], B=p[3:6])
            o.set_spins(Ss[r])
            tot += wr * o.energy()
        return tot

    p0 = np.array([1.0, 0.1, -0.05, 0.2, 0.0, 0.0])
    for k in range(6):
        dp = np.zeros(6)
        dp[k] = h
        fd = (loss(p0 + dp) - loss(p0 - dp)) / (2 * h)
        assert params.grad[k].item() == pytest.approx(fd, rel=2e-3, abs=2e-4), k
    # spin gradient: d e_r / d S_i = (h_i - B)/Nc
    o = oracle.System(L, **C4)
    o.set_spins(Ss[1])
    ref = -0.5 * (o.local_fields() - np.array(C4["B"])) / L ** 3
    got = spins.grad[g.N():, :3].cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("L", [2, 3])
def test_ssf_backward_matches_finite_differences(L):
    g = pc.pyrochlore_system(L, n_replicas=2, J1=1.0)
    corr = ["zz", "xy", "yz"]
    g.ssf_configure(corr, 0, [])
    rng = np.random.default_rng(L)
    for r in range(2):
        g.set_spins(unit(rng, g.N()), r)
    spins = ag.spins_tensor(g).clone().requires_grad_(True)
    nk = L ** 3
    w = torch.as_tensor(rng.uniform(0, 1, (2, 3, nk, 2)), device="cuda")
    tgt = torch.as_tensor(rng.normal(0, 10, (2, 3, nk, 2)), device="cuda")
    S = ag.ssf(g, spins)
    loss = (w * (S - tgt) ** 2).sum()
    loss.backward()
    grad = spins.grad[:, :3].cpu().numpy()
    Ss = [g.spins(0), g.spins(1)]
    wn, tn = w.cpu().numpy(), tgt.cpu().numpy()

    def L_of(r, Sr):
        o = oracle.System(L)
        o.set_spins(Sr)
        Sq = o.ssf(corr)
        return float((wn[r] * (Sq - tn[r]) ** 2).sum())

    h = 1e-4
    scale = np.abs(grad).max()
    for r in range(2):
        for i in rng.choice(g.N(), 6, replace=False):
            for a in range(3):
                Sp = Ss[r].copy()
                Sp[i, a] += h
                lp = L_of(r, Sp)
                Sp[i, a] -= 2 * h
                lm = L_of(r, Sp)
                fd = (lp - lm) / (2 * h)
                got = grad[r * g.N() + i, a]
                assert abs(got - fd) <= 2e-3 * scale, (r, i, a, got, fd)


def test_ssf_forward_batched_matches_current():
    g = pc.pyrochlore_system(4, n_replicas=3, J1=1.0)
    g.ssf_configure(["xx", "zz", "xz"], 1, [4])
    g.random_spins(5)
    out = torch.empty((3, 3, 64, 2), dtype=torch.float64, device="cuda")
    g.ssf_forward_device(out.data_ptr())
    for r in range(3):
        np.testing.assert_allclose(out[r].cpu().numpy(), g.ssf_current(r), rtol=0, atol=1e-9)


def test_gradient_quench_reaches_luttinger_tisza_bound():
    L = 2
    for c in (dict(J1=1.0), dict(J1=1.0, J2=-0.1, J3=0.05)):
        g = pc.pyrochlore_system(L, n_replicas=4, **c)
        g.random_spins(3)
        hist = ag.gradient_quench(g, steps=500, lr=0.05)
        e_lt, _ = oracle.lt.lt_minimum(L, c["J1"], c.get("J2", 0.0), c.get("J3", 0.0))
        e_spin = hist[-1] / 16
        assert (e_spin >= e_lt - 1e-5).all()  # LT is a lower bound
        assert (np.diff(hist, axis=0) <= 1e-4).all()  # descent
        if "J2" not in c:
            # J1 only: the bound -1 per spin is reached (zero tetrahedron sums)
            assert (e_spin <= e_lt + 0.02).all(), e_spin


# ----------------------------------------------------------------- tempering
def test_pt_bookkeeping():
    Ls = [2, 2, 2, 2, 3, 3, 3]
    # closely spaced ladders so that exchanges are accepted often
    T = [1.0, 0.95, 0.9, 0.85, 1.0, 0.95, 0.9]
    g = pc.pyrochlore_system(Ls, J1=1.0, J3=0.02, B=(0, 0, 0.1), seed=3)
    g.random_spins(1)
    g.pt_configure(T)
    g.ssf_configure(["xx", "yy", "zz"], 7, [2, 2, 2, 2, 3, 3, 3])
    g.pt_run(40, 5, 10)
    Ts, E, E2, n = g.pt_energy()
    assert list(Ts) == T
    assert np.isfinite(E).all() and np.isfinite(E2).all()
    assert (n == 40).all()
    assert (E2 / n >= (E / n) ** 2 - 1e-9).all()
    att, acc = g.pt_exchange_stats()
    # pairs (0,1),(2,3) even rounds, (1,2) odd rounds within each ladder
    assert list(att[:4]) == [20, 20, 20, 0] and list(att[4:]) == [20, 20, 0]
    assert (acc <= att).all() and acc.sum() > 0
    slots = g.pt_slots()
    assert sorted(slots[:4]) == [0, 1, 2, 3] and sorted(slots[4:]) == [4, 5, 6]
    s, q, ns = g.ssf_read(3, 2)
    assert ns == 20 and s[..., 0].min() >= -1e-6


def _stats_compare(a_mean, a_err, b_mean, b_err, what):
    z = np.abs(a_mean - b_mean) / np.sqrt(a_err ** 2 + b_err ** 2 + 1e-300)
    frac = np.mean(z <= 3)
    assert frac >= 0.95 and z.max() <= 5, (what, frac, z.max(), np.argmax(z))
    return z


@pytest.mark.parametrize("schedule", [0, 1])
def test_pt_equilibrium_matches_reference_tempering(schedule):
    """Batched GPU tempering vs the oracle's temper.cpp emulation (equilibrium
    <e>(T) per slot, batch-mean errors over K = 32 independent runs per side,
    the ensemble size of the statistical protocol; with 16 runs the error
    estimates themselves scatter enough that a 3-sigma cut on 5 temperatures
    fails about one stream in a hundred); for both sweep schedules."""
    L, T = 2, [2.0, 1.2, 0.8, 0.5, 0.3]
    c = dict(J1=1.0, J2=0.0, J3=0.02, B=(0, 0, 0.1))
    K = 32
    gpu_means = []
    for k in range(K):
        s = pc.pyrochlore_system(L, n_replicas=len(T), seed=100 + k, schedule=schedule, **c)
        s.random_spins(k)
        s.pt_configure(T)
        s.pt_run(40, 5)  # burn-in
        s.pt_reset_stats()
        s.pt_run(200, 5)
        _, E, _, n = s.pt_energy()
        gpu_means.append(E / n)
    gpu_means = np.array(gpu_means)

    def run(k):
        es, e2, att, acc = oracle.temper(L, T, seed=1000 + 7 * k, n_burn_in=0, n_burn_rounds=40, n_rounds=200,
                                         n_sweep=5, **c)
        return es / 200

    with cf.ThreadPoolExecutor(8) as ex:
        cpu_means = np.array(list(ex.map(run, range(K))))
    _stats_compare(gpu_means.mean(0), gpu_means.std(0, ddof=1) / np.sqrt(K), cpu_means.mean(0),
                   cpu_means.std(0, ddof=1) / np.sqrt(K), "pt <e>")


@pytest.mark.parametrize("schedule", [0, 1])
def test_anneal_config1_statistical_parity(schedule):
    """The plain anneal of config 1 (L=4, J1=1, T 10 -> 0.05 over 100 log steps,
    16 sweeps per step, S(q) xx/yy/zz at T in {1, 0.1, 0.05} from 64 samples,
    16 burn-in sweeps, uniform start): <e>(T), the cross-seed C_v and S(q) of K
    GPU seeds (batched replicas) against K seeds of the reference-faithful
    oracle (Xoroshiro128++, sequential sweep)."""
    from pyro_cmc_b200.anneal import anneal_batch

    K = 32
    args = dict(L=4, J1=1.0, J2=0.0, J3=0.0, B=(0, 0, 0), T_hot=10.0, T_cold=0.05, T_sample=[1.0, 0.1, 0.05],
                n_steps=100, n_sweep=16, n_burn_in=16, n_sample=64, corr=["xx", "yy", "zz"])
    res = anneal_batch(K=K, seed=0xdeadbeef, schedule=schedule, **args)
    e_gpu = res["e"]  # [K, n_T]

    def run(k):
        o = oracle.System(4, J1=1.0, seed=0xdeadbeef + 7919 * k)
        o.random_spins(17 + k)
        T, e, ssum, ssq = o.anneal(10.0, 0.05, [1.0, 0.1, 0.05], 100, 16, 16, 64, ["xx", "yy", "zz"])
        return T, e, ssum

    with cf.ThreadPoolExecutor(8) as ex:
        out = list(ex.map(run, range(K)))
    T_cpu = out[0][0]
    np.testing.assert_allclose(res["T"], T_cpu, rtol=1e-14)
    e_cpu = np.array([o[1] for o in out])
    _stats_compare(e_gpu.mean(0), e_gpu.std(0, ddof=1) / np.sqrt(K), e_cpu.mean(0),
                   e_cpu.std(0, ddof=1) / np.sqrt(K), "<e>")
    # cross-seed C_v (plot_ssf.py:181-186 with one sample per seed): error by jackknife
    def cv(e):
        return e.var(0, ddof=1) / T_cpu ** 2

    def jk(e):
        vals = np.array([cv(np.delete(e, i, 0)) for i in range(len(e))])
        return np.sqrt((len(e) - 1) * vals.var(0))

    _stats_compare(cv(e_gpu), jk(e_gpu), cv(e_cpu), jk(e_cpu), "C_v")
    # S(q) per sample at the sample temperatures (real part of the diagonal correlators)
    s_gpu = res["ssf_sum"][..., 0] / 64  # [K, nT, corr, nk]
    s_cpu = np.array([o[2][..., 0] for o in out]) / 64
    # the reference writes T_sample slots ascending; anneal_batch returns them in visit
    # order (descending), as does the oracle
    _stats_compare(s_gpu.mean(0).ravel(), (s_gpu.std(0, ddof=1) / np.sqrt(K)).ravel(),
                   s_cpu.mean(0).ravel(), (s_cpu.std(0, ddof=1) / np.sqrt(K)).ravel(), "S(q)")


@pytest.mark.parametrize("L", [8, 11, 16, 64])
def test_ssf_backward_large_L_matches_fft_adjoint(L):
    """The S(q) backward at sizes beyond finite differences: L = 11 (runtime
    line length), 8, 16 and 64 (the instantiated sizes; 16 and 64 with the
    swizzled shared layout), against the numpy-FFT adjoint of
    ssf_manager::sample."""
    from oracle import ssf_fft
    corr = ["xx", "yy", "zz", "xy", "xz", "yz", "zx"]
    g = pc.pyrochlore_system(L, J1=1.0)
    g.ssf_configure(corr, 0, [])
    g.random_spins(L)
    spins = ag.spins_tensor(g).clone().requires_grad_(True)
    rng = np.random.default_rng(L)
    nk = L ** 3
    D = rng.normal(size=(1, len(corr), nk, 2))
    S = ag.ssf(g, spins)
    (S * torch.as_tensor(D, device="cuda")).sum().backward()
    got = spins.grad[:, :3].cpu().numpy()
    ref = ssf_fft.adjoint(g.spins(), L, corr, D[0])
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-5 * scale * max(1.0, np.log2(nk)), np.abs(got - ref).max() / scale


def _lt_matrix(L, K, J1, J2, J3, Delta):
    """The oracle's LT matrix M(k) (oracle/lt.py bonds) at one K, numpy."""
    import oracle.lt as olt
    sysd = oracle.System(1, J1=1.0, J2=1.0, J3=1.0, j1_mode=1)
    tables = {k: [sysd.spec_displacements(spec, p) for p in range(4)] for k, spec in
              (("J1", 0), ("J2", 1), ("J3a", 2), ("J3b", 3))}
    r = np.array([olt.LINK[s % 4] + olt.FCC[s // 4] for s in range(16)])
    rmod = {tuple(x % 8): s for s, x in enumerate(r)}
    z = olt.LINK / np.sqrt(3.0)
    k = 2 * np.pi * np.asarray(K) / (8.0 * L)
    Mk = np.zeros((48, 48), complex)
    for name, j in (("J1", J1), ("J2", J2), ("J3a", J3), ("J3b", J3)):
        if j == 0.0:
            continue
        for a in range(16):
            for d in tables[name][a % 4]:
                b = rmod[tuple((r[a] + d) % 8)]
                M = j * (np.eye(3) + (Delta - 1.0) * np.outer(z[a % 4], z[b % 4])) if name == "J1" else j * np.eye(3)
                Mk[3 * a:3 * a + 3, 3 * b:3 * b + 3] += M * np.exp(1j * (k @ np.asarray(d, float)))
    return Mk


@pytest.mark.parametrize("L,J", [(2, (1.0, 0.0, 0.0, 1.0)), (3, (1.0, 0.1, -0.05, 0.5)),
                                 (4, (-0.7, 0.3, 0.02, 1.3)), (4, (1.0, -0.1, 0.05, 1.0))])
def test_lt_on_gpu_matches_oracle(L, J):
    """pc_lt_minimum against the numpy restatement of src/luttinger_tisza.cpp:
    the eigenvalue map at every k (FP64 eigvalsh), E_min and k*, and the
    eigenvector (M v = lambda v, unit norm)."""
    import oracle.lt as olt
    from pyro_cmc_b200.lt import lt_minimum
    J1, J2, J3, D = J
    res = lt_minimum(L, J1, J2, J3, D)
    e_ref, k_ref = olt.lt_minimum(L, J1, J2, J3, D)
    assert abs(res["E_min"] - e_ref) <= 1e-9 * max(1.0, abs(e_ref))
    lam = res["eigenvalue_map"]
    for K in [(0, 0, 0), tuple(res["k_star_idx"]), (1, 0, L - 1), (L - 1, L // 2, 1)]:
        Mk = _lt_matrix(L, K, J1, J2, J3, D)
        assert abs(lam[K] - np.linalg.eigvalsh(Mk)[0]) <= 1e-9 * max(1.0, np.abs(Mk).max())
    assert abs(lam[tuple(k_ref)] - 2 * e_ref) <= 1e-9 * max(1.0, abs(e_ref))
    v = res["eigenvector"]
    Mk = _lt_matrix(L, tuple(res["k_star_idx"]), J1, J2, J3, D)
    assert abs(np.linalg.norm(v) - 1.0) < 1e-9
    assert np.linalg.norm(Mk @ v - 2 * res["E_min"] * v) <= 1e-6 * max(1.0, np.abs(Mk).max())


def test_seed_merge_on_device_matches_acc_runs():
    """anneal_batch(merge=True): the device merge of K seeds (pc_ssf_merge)
    against the restatement of scripts/acc_runs.py (pinned on the reference's
    own outputs) applied to the per-seed accumulators."""
    from oracle import merge as om
    from pyro_cmc_b200.anneal import anneal_batch
    corr = ["xx", "yy", "zz", "xy", "xz", "yz"]
    K = 4
    r = anneal_batch(K=K, L=3, J1=1.0, J2=-0.1, J3=0.05, T_hot=5.0, T_sample=[0.3, 0.1], n_steps=6, n_sweep=3,
                     n_burn_in=3, n_sample=5, corr=corr, seed=8, merge=True)
    # per-seed arrays in acc_runs layout: [K, n_corr, n_T, n_k, 2]
    sc = np.transpose(r["ssf_sum"], (0, 2, 1, 3, 4))
    sc2 = np.transpose(r["ssf_sq"], (0, 2, 1, 3, 4))
    n = np.tile(r["n_ssf"].astype(float), (K, 1))
    ref = om.merge_ssf(sc, sc2, n)
    for t, m in enumerate(r["merged"]["ssf"]):
        for k in ("static_corr", "static_corr_2", "var_inter", "var_intra"):
            a, b = m[k], ref[k][:, t]
            assert np.abs(a - b).max() <= 1e-12 * max(1.0, np.abs(b).max()), k
        for s in range(K):
            p = om.plane_invariants(sc[s][:, t:t + 1], n[s][t:t + 1], corr)
            np.testing.assert_allclose(m["w"][s], p["w"][0], atol=1e-9)
            np.testing.assert_allclose(m["chi_frac"][s], p["chi_frac"][0], atol=1e-9)
            np.testing.assert_allclose(m["tr"][s], p["tr"][0], rtol=1e-12, atol=1e-9)
    e = om.merge_energy(r["e"], r["e"] ** 2, np.ones_like(r["e"]))
    np.testing.assert_allclose(r["merged"]["energy"]["var"], e["var"], rtol=1e-12, atol=1e-12)
