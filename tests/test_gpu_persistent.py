"""Tempering rounds in one persistent cooperative launch (pc_set_pt_persistent)
against the per-pass graph schedule of the same rounds: uneven-L ladders
(src/temper.cpp:418-474 per ladder), both sweep schedules, the three coupling
kinds the structured kernels distinguish (all isotropic; isotropic with J2 = 0;
XXZ J1). The site updates and draws are the same, so the spins, the slot
assignment and the exchange statistics are identical; the energy samples
(the same per-cell sums, the per-replica FP64 sums in another order) agree to
1e-5 relative. Then: S(q) samples taken
between the launches, the sweep and round counters carried on by the per-pass
path, and the bounded grid-barrier wait running out (PC_ERR_TIMEOUT) with the
system usable afterwards."""
import numpy as np
import pytest

import pyro_cmc_b200 as pc
from pyro_cmc_b200 import _lib

pytestmark = pytest.mark.gpu

CASES = [
    dict(J1=1.0, J2=-0.1, J3=0.05, B=(0.0, 0.0, 0.1)),             # every group j I
    dict(J1=1.0, J2=0.0, J3=0.02, B=(0.0, 0.0, 0.1)),              # j I, J2 group zero
    dict(J1=1.0, J2=0.1, J3=0.05, Delta=0.6, B=(0.1, 0.0, 0.3)),   # XXZ J1: general matrices
]
LS = [4] * 4 + [6] * 3 + [8] * 4
# closely spaced ladders: swaps are accepted, so later sweeps run at exchanged
# temperatures (written by block 0, read by every block of the next phase)
TS = [1.0, 0.99, 0.98, 0.97, 1.0, 0.99, 0.98, 1.0, 0.995, 0.99, 0.985]


def _pair(Ls, T, c, schedule, seed, threads=None):
    out = []
    for persistent in (False, True):
        s = pc.pyrochlore_system(Ls, seed=seed, schedule=schedule, **c)
        if threads:
            s.set_tile(threads, 4)
        s.random_spins(seed)
        s.pt_configure(T)
        if persistent:
            s.set_pt_persistent(True)
            assert s.pt_persistent()
        out.append(s)
    return out


def _same_chain(a, b, R):
    for r in range(R):
        np.testing.assert_array_equal(a.spins(r), b.spins(r))
    np.testing.assert_array_equal(a.pt_slots(), b.pt_slots())
    for x, y in zip(a.pt_exchange_stats(), b.pt_exchange_stats()):
        np.testing.assert_array_equal(x, y)
    _, Ea, E2a, na = a.pt_energy()
    _, Eb, E2b, nb = b.pt_energy()
    np.testing.assert_array_equal(na, nb)
    np.testing.assert_allclose(Eb, Ea, rtol=1e-5, atol=1e-5 * np.abs(Ea).max())
    np.testing.assert_allclose(E2b, E2a, rtol=1e-5, atol=1e-5 * np.abs(E2a).max())
    assert a.sweep_counter() == b.sweep_counter()


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_persistent_rounds_give_the_per_pass_chain(schedule, ci):
    a, b = _pair(LS, TS, CASES[ci], schedule, 7 + ci)
    for s in (a, b):
        s.pt_run(6, 3)
    _same_chain(a, b, len(LS))
    att, acc = b.pt_exchange_stats()
    assert att.sum() > 0 and acc.sum() > 0
    # the counters the persistent launch advanced carry on in the per-pass path
    b.set_pt_persistent(False)
    for s in (a, b):
        s.pt_run(2, 3)
    _same_chain(a, b, len(LS))


@pytest.mark.parametrize("threads", [64, 128])
def test_persistent_rounds_other_block_sizes(threads):
    a, b = _pair(LS, TS, CASES[0], 1, 11, threads=threads)
    for s in (a, b):
        s.pt_run(4, 2)
    _same_chain(a, b, len(LS))


def test_persistent_rounds_with_ssf_samples():
    """ssf_every = 3 with 5 sweeps per round: samples fall at different
    sweeps of successive rounds, once after a round's last sweep (before its
    energies and exchange); every slot's S(q) accumulators match exactly."""
    Ls = [2, 2, 2, 2, 3, 3, 3]
    T = [1.0, 0.95, 0.9, 0.85, 1.0, 0.95, 0.9]
    a, b = _pair(Ls, T, CASES[1], 1, 3)
    for s in (a, b):
        s.ssf_configure(["xx", "yy", "zz", "xy"], 7, Ls)
        s.pt_run(9, 5, 3)
    _same_chain(a, b, len(Ls))
    for slot, L in enumerate(Ls):
        sa, qa, na = a.ssf_read(slot, L)
        sb, qb, nb = b.ssf_read(slot, L)
        assert na == nb == 15
        np.testing.assert_array_equal(sa, sb)
        np.testing.assert_array_equal(qa, qb)


def test_persistent_barrier_wait_runs_out_and_system_recovers():
    """With the wait bound at zero polls the first block to reach a grid
    barrier stops waiting at once, sets the device error flag, and every block
    leaves at its next barrier: PC_ERR_TIMEOUT, no fault. The same system then
    runs rounds normally."""
    Ls = [16] * 8
    T = list(np.linspace(1.0, 0.3, 8))
    s = pc.pyrochlore_system(Ls, seed=5, schedule=1, **CASES[0])
    s.random_spins(5)
    s.pt_configure(T)
    s.set_pt_persistent(True)
    s.set_wait_limit(0)
    with pytest.raises(pc.PyroCMCError) as ei:
        s.pt_run(2, 2)
    assert ei.value.code == _lib.ERR_TIMEOUT and "grid barrier" in str(ei.value)
    s.set_wait_limit(-1)
    s.pt_reset_stats()
    s.pt_run(3, 2)
    _, E, _, n = s.pt_energy()
    assert (n == 3).all() and np.isfinite(E).all()
    for r in range(len(Ls)):
        S = s.spins(r)
        np.testing.assert_allclose(np.linalg.norm(S, axis=1), 1.0, atol=1e-5)


def test_persistent_rounds_refused_where_not_covered():
    s = pc.pyrochlore_system([4, 4], seed=1, update=1, **CASES[0])
    s.pt_configure([1.0, 0.5])
    with pytest.raises(pc.PyroCMCError) as ei:
        s.set_pt_persistent(True)
    assert ei.value.code == _lib.ERR_UNSUPPORTED
    s = pc.pyrochlore_system([4, 4], seed=1, overrelax_mode=1, **CASES[0])
    with pytest.raises(pc.PyroCMCError) as ei:
        s.set_pt_persistent(True)
    assert ei.value.code == _lib.ERR_UNSUPPORTED


def test_persistent_rounds_at_the_batched_workload():
    """The batched tempering form at full size (128 replicas, L = 8, 12, 16,
    24 with 32 temperatures each, J = (1, 0, 0.02), B = (0, 0, 0.1), the fused
    schedule), 3 rounds of 10 sweeps with S(q) every 16: ~1000 resident blocks
    gather neighbours that other blocks wrote one barrier earlier. Spins,
    slots, exchange statistics and S(q) accumulators identical to the per-pass
    graphs."""
    Ls = [8] * 32 + [12] * 32 + [16] * 32 + [24] * 32
    T = np.concatenate([np.geomspace(2.0, 0.02, 32)] * 4)
    c = dict(J1=1.0, J2=0.0, J3=0.02, B=(0.0, 0.0, 0.1))
    a, b = _pair(Ls, T, c, 1, 7)
    for s in (a, b):
        s.ssf_configure(["xx", "yy", "zz"], len(Ls), sorted(Ls))
        s.pt_run(3, 10, 16)
    _same_chain(a, b, len(Ls))
    for slot in (0, 40, 70, 127):
        L = sorted(Ls)[slot]
        for x, y in zip(a.ssf_read(slot, L), b.ssf_read(slot, L)):
            np.testing.assert_array_equal(np.asarray(x), np.asarray(y))


def test_autotune_after_configure_keeps_the_ladder():
    """pc_autotune times its candidates at T = 1 on the system itself; it puts
    back the spins, the sweep counter and the temperatures (the ladder's
    current assignment), so a tempering run autotuned after pc_pt_configure
    is the chain of the same run without autotuning (the chain does not
    depend on the tile the autotuner picks)."""
    c = CASES[0]
    runs = []
    for tune in (False, True):
        s = pc.pyrochlore_system(LS, seed=21, schedule=1, **c)
        s.random_spins(21)
        s.pt_configure(TS)
        s.pt_run(1, 2)
        if tune:
            s.autotune()
        s.pt_run(3, 2)
        runs.append(s)
    _same_chain(runs[0], runs[1], len(LS))
