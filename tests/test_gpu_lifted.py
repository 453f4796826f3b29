"""Lifted Metropolis on the GPU (sweep_lifted_Metropolis, src/MC.cpp:194-302):
site by site against the oracle's Philox mirror, statistically against
standard Metropolis with the reference's own acceptance test
(test/bench_lifted.cpp), and through the anneal driver's --lifted flag."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import pyro_cmc_b200 as pc
from pyro_cmc_b200 import build
from pyro_cmc_b200.anneal import anneal_batch

pytestmark = pytest.mark.gpu

COUP = dict(J1=1.0, J2=0.1, J3=-0.05, Delta=0.5, B=(0.2, 0.0, 0.0))


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def dirs_of(g):
    return np.where(g.spins_f4()[:, 3] < 0, -1, 1).astype(np.int8)


@pytest.mark.parametrize("update", [1, 2])
@pytest.mark.parametrize("path", ["generic", "v0", "v3"])
@pytest.mark.parametrize("T", [0.3, 2.0])
def test_lifted_sweeps_follow_oracle_mirror(update, path, T):
    seed = 4242
    g = pc.pyrochlore_system(3, seed=seed, generic=(path == "generic"), schedule=1, update=update, **COUP)
    if path != "generic":
        g.set_load_variant(int(path[1]))
    o = oracle.System(3, seed=seed, **COUP)
    rng = np.random.default_rng(7)
    g.set_spins(unit(rng, o.N))
    o.set_spins(g.spins())
    _, col = g.colours()
    flips = 0
    for sweep in range(4):
        acc_g = g.sweep(T, 1, 1)[0]
        acc_o = o.sweep_philox(T, seed, 0, sweep, col, n_overrelax=1, or_mode=0, fused=True, update=update)
        assert int(acc_g) == int(acc_o)
        np.testing.assert_allclose(g.spins(), o.spins(), atol=1e-4)
        d = dirs_of(g)
        np.testing.assert_array_equal(d, o.lifted_dirs())
        flips += int((d < 0).sum())
        o.set_spins(g.spins())
    assert 0 < int(acc_g) < o.N and flips > 0  # both branches exercised


def _energies(update, seed, K=64, L=4, T=0.5, n_burn=400, n_sample=60, every=5):
    g = pc.pyrochlore_system(L, J1=-1.0, J2=0.3, seed=seed, n_replicas=K, update=update)
    g.random_spins(seed + 1)
    g.sweep(T, n_burn, 1, count=False)
    e = np.empty((n_sample, K))
    for i in range(n_sample):
        g.sweep(T, every, 1, count=False)
        e[i] = g.energy()[0] / 16.0  # per spin
    return e


@pytest.mark.parametrize("update", [1, 2])
def test_lifted_samples_like_metropolis(update):
    """test/bench_lifted.cpp:240-272 on the pyrochlore lattice: J1 = -1,
    J2 = 0.3, T = 0.5; |<E>_std - <E>_lifted| and |<E^2>_std - <E^2>_lifted|
    per spin below 0.1 min(|J1|, |J2|), and within 5 sigma (replica spread)."""
    a = _energies(0, 3)
    b = _energies(update, 5)
    tol = 0.1 * min(1.0, 0.3)
    ma, mb = a.mean(axis=0), b.mean(axis=0)  # per-replica time averages
    sa = ma.std(ddof=1) / np.sqrt(len(ma))
    sb = mb.std(ddof=1) / np.sqrt(len(mb))
    assert abs(ma.mean() - mb.mean()) < tol
    assert abs((a ** 2).mean() - (b ** 2).mean()) < tol
    assert abs(ma.mean() - mb.mean()) < 5 * np.hypot(sa, sb) + 1e-4, (ma.mean(), mb.mean(), sa, sb)


def test_anneal_driver_lifted_matches_python_protocol(tmp_path):
    build.build()
    args = ["-o", tmp_path, "-s", 91, 2, "--J1", 1, "--J2", -0.1, "--J3", 0.05, "--T_sample", 0.5,
            "--n_steps", 8, "--n_sweep", 4, "--n_burn_in", 4, "--n_sample", 2, "--init_uniform", "--lifted",
            "--correlators", "xx"]
    r = subprocess.run([os.path.join(build.BIN, "anneal"), *map(str, args)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "(lifted Metropolis)" in r.stdout
    files = [f for f in os.listdir(tmp_path) if f.endswith(".out.h5")]
    from pyro_cmc_b200.h5compat import File
    with File(os.path.join(tmp_path, files[0])) as f:
        E = f["/energy/E"][:]
    py = anneal_batch(K=1, L=2, J1=1, J2=-0.1, J3=0.05, T_hot=10.0, T_sample=[0.5], n_steps=8, n_sweep=4,
                      n_burn_in=4, n_sample=2, corr=["xx"], seed=91, init_seed=91 ^ 0x5EED, update=1)
    np.testing.assert_array_equal(py["e"][0], E)
    std = anneal_batch(K=1, L=2, J1=1, J2=-0.1, J3=0.05, T_hot=10.0, T_sample=[0.5], n_steps=8, n_sweep=4,
                       n_burn_in=4, n_sample=2, corr=["xx"], seed=91, init_seed=91 ^ 0x5EED, update=0)
    assert not np.array_equal(std["e"][0], E)  # the flag changes the chain
