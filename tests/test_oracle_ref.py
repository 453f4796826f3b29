"""The oracle pinned on the reference's own Monte Carlo code (no GPU).

oracle/_ref/libref_mc.so is the reference's src/MC.cpp compiled unchanged
(oracle/make_ref.sh, with the lattice_lib / HDF5 stand-ins of oracle/ref_shim/).
These tests check the oracle's restatement (oracle/pyro_oracle.cpp) against
it: lattice positions and bond shells exactly; energy per cell and local field
to FP64 rounding; and whole sequential chains -- Metropolis + overrelaxation
(src/MC.cpp:111-163), lifted u-form (:249-291) and lifted rotation form
(:194-302) -- from the same Xoroshiro128++ seed, with identical accepted counts
and lifting directions after every sweep. The two sum a shell's neighbours in
different orders (the oracle derives its displacement tables from the geometry,
the reference lists them by hand), so the spins differ by FP64 rounding, which
a chain amplifies slowly; the tolerance grows with the sweep count.

The committed fixture tests/golden/ref_mc_chains.npz (made by
tests/golden/make_ref_mc_golden.py from the same library) carries the pin
where the library is not built.
"""
import os

import numpy as np
import pytest

import oracle
from oracle import ref

GOLD = os.path.join(os.path.dirname(__file__), "golden")
needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref/libref_mc.so not built (needs the reference tree)")

COUPLINGS = [
    dict(J1=1.0, J2=0.0, J3=0.0, Delta=1.0, B=(0.0, 0.0, 0.0)),
    dict(J1=1.0, J2=-0.1, J3=0.05, Delta=1.0, B=(0.0, 0.0, 0.0)),  # anneal, L = 16
    dict(J1=1.0, J2=0.0, J3=0.02, Delta=1.0, B=(0.0, 0.0, 0.1)),  # tempering ladders
    dict(J1=1.0, J2=0.1, J3=-0.05, Delta=1.0, B=(0.2, 0.0, 0.0)),  # differentiable form
    dict(J1=1.0, J2=0.1, J3=0.05, Delta=1.0, B=(0.0, 0.0, 0.5)),  # field-cool, L = 64
    dict(J1=-1.0, J2=0.3, J3=-0.02, Delta=0.6, B=(0.1, 0.2, 0.3)),  # XXZ
]


def _spins(N, seed):
    rng = np.random.default_rng(seed)
    S = rng.normal(size=(N, 3))
    return S / np.linalg.norm(S, axis=1, keepdims=True)


@needs_ref
@pytest.mark.parametrize("L", [1, 2, 3])
def test_positions_and_bond_shells_match_reference(L):
    c = COUPLINGS[5]
    r = ref.RefSystem(L, **c)
    o = oracle.System(L, **c)
    pos_o, _ = o.positions()
    assert (r.positions() == pos_o).all()
    # the oracle's shells, rebuilt from its per-spec neighbour lists with
    # setup_lattice's split (src/MC.cpp:28-50): own pyro_sl <= other's -> J
    psl = np.arange(r.N) // (L ** 3) % 4
    want = [[] for _ in range(r.N)]
    for spec in range(o.num_specs()):
        J = o.spec_matrix(spec)
        nb = o.neighbours(spec, 16)
        for i in range(r.N):
            js = [j for j in nb[i] if j >= 0]
            src = sorted(j for j in js if psl[i] <= psl[j])
            tgt = sorted(j for j in js if psl[i] > psl[j])
            if src:
                want[i].append((J, src))
            if tgt:
                want[i].append((J.T, tgt))
    got = r.shells()
    for i in range(r.N):
        assert len(got[i]) == len(want[i]), i
        for (Jg, ng), (Jw, nw) in zip(got[i], want[i]):
            assert sorted(ng.tolist()) == nw
            np.testing.assert_allclose(Jg, Jw, rtol=0, atol=1e-15)


@needs_ref
@pytest.mark.parametrize("ci", range(len(COUPLINGS)))
@pytest.mark.parametrize("L", [1, 2, 4, 8])
def test_energy_and_local_field_match_reference(L, ci):
    c = COUPLINGS[ci]
    r = ref.RefSystem(L, **c)
    o = oracle.System(L, **c)
    S = _spins(r.N, 100 + L)
    r.set_spins(S)
    o.set_spins(S)
    assert abs(r.energy() - o.energy()) <= 1e-13 * 16 * 8
    np.testing.assert_allclose(o.local_fields(), r.local_fields(), rtol=0, atol=1e-13)


@needs_ref
@pytest.mark.parametrize("L", [12, 16])
def test_energy_and_local_field_match_reference_at_config_sizes(L):
    c = COUPLINGS[1]
    r = ref.RefSystem(L, **c)
    o = oracle.System(L, **c)
    S = _spins(r.N, 7)
    r.set_spins(S)
    o.set_spins(S)
    assert abs(r.energy() - o.energy()) <= 1e-13 * 16 * 8
    np.testing.assert_allclose(o.local_fields(), r.local_fields(), rtol=0, atol=1e-13)


@needs_ref
@pytest.mark.parametrize("mode", ["std", "u", "rot"])
@pytest.mark.parametrize("ci", [1, 4, 5])
def test_sequential_chains_match_reference(mode, ci):
    c = COUPLINGS[ci]
    L, seed, T = 4, 31 + ci, 0.4
    r = ref.RefSystem(L, seed=seed, **c)
    o = oracle.System(L, seed=seed, **c)
    S = _spins(r.N, seed)
    r.set_spins(S)
    o.set_spins(S)
    for k in range(6):
        if mode == "std":
            a, b = r.sweep(T, 1, 1), o.sweep(T, 1, 1)
        else:
            a, b = r.sweep_lifted(T, 1, 1, rot=mode == "rot"), o.sweep_lifted(T, 1, 1, rot=mode == "rot")
        assert a == b, (k, a, b)
        assert (r.lifted_dirs() == o.lifted_dirs()).all(), k
        assert np.abs(r.spins() - o.spins()).max() <= 1e-12 * 10 ** k, k


def test_oracle_matches_committed_reference_chains():
    """Same pin from tests/golden/ref_mc_chains.npz (no reference build needed)."""
    import sys
    sys.path.insert(0, GOLD)
    import make_ref_mc_golden as mk  # the cases the fixture was made from

    g = np.load(os.path.join(GOLD, "ref_mc_chains.npz"))
    for name, L, c, seed, T in mk.CASES:
        o = oracle.System(L, seed=seed, **c)
        S0 = g[name + "/S0"]
        o.set_spins(S0)
        assert abs(o.energy() - float(g[name + "/energy"])) <= 1e-13 * 16 * 8
        np.testing.assert_allclose(o.local_fields(), g[name + "/field"], rtol=0, atol=1e-13)
        for mode in ("std", "u", "rot"):
            o = oracle.System(L, seed=seed, **c)
            o.set_spins(S0)
            for k in range(mk.N_SWEEPS):
                if mode == "std":
                    a = o.sweep(T, 1, 1)
                else:
                    a = o.sweep_lifted(T, 1, 1, rot=mode == "rot")
                assert a == int(g[f"{name}/{mode}/accepted"][k]), (name, mode, k)
                assert (o.lifted_dirs() == g[f"{name}/{mode}/dirs"][k]).all()
                assert np.abs(o.spins() - g[f"{name}/{mode}/spins"][k]).max() <= 1e-12 * 10 ** k
