"""Cluster-resident sweeps (pc_set_cluster_sweeps) against the per-pass
colour kernels, through the C ABI: one thread-block cluster per replica runs
every colour pass of a sweep call in one launch with the lattice in
distributed shared memory. Same passes, draws and move arithmetic in a
separately compiled function, so the two chains agree up to rounding (FMA
contraction can differ between the two compilations): after one sweep, 99.5 %
of the spin components within 1e-5 and all within 1e-3, the accepted-move
counts within 0.1 %, the sweep counters equal; a cluster sweep followed by a
per-pass sweep continues the chain (sweep counter and draws). Covered: the fused
and the reference-order schedules, both overrelaxation forms, one and four
sublattices per colour class, one and several replicas, L from 3 to 16.
"""
import numpy as np
import pytest

import pyro_cmc_b200 as pc
from pyro_cmc_b200 import _lib

pytestmark = pytest.mark.gpu

J3ON = dict(J1=1.0, J2=0.1, J3=0.05, Delta=0.8, B=(0.0, 0.1, 0.5))  # 16 colour classes
J3OFF = dict(J1=1.0, J2=-0.1, J3=0.0, Delta=1.0, B=(0.2, 0.0, 0.0))  # 4 classes of 4 sublattices


def _close_rounding(a, b):
    d = np.abs(np.asarray(a, float) - np.asarray(b, float))
    assert (d <= 1e-5).mean() >= 0.995, (d <= 1e-5).mean()
    assert d.max() <= 1e-3, d.max()


def _pair(L, R, c, schedule, or_mode):
    out = []
    for cluster in (False, True):
        s = pc.pyrochlore_system(L, n_replicas=R, seed=77, schedule=schedule, overrelax_mode=or_mode, **c)
        s.random_spins(5)
        if cluster:
            s.set_cluster_sweeps(True)
            assert s.cluster_sweeps()
        out.append(s)
    return out


@pytest.mark.parametrize("L,R,c,schedule,or_mode,n_or", [
    (16, 1, J3ON, 1, 0, 1),
    (16, 1, J3ON, 0, 0, 2),
    (8, 3, J3ON, 1, 1, 1),
    (8, 2, J3OFF, 0, 1, 1),
    (4, 2, J3ON, 1, 0, 2),
    (3, 1, J3OFF, 1, 0, 1),
    (12, 1, J3ON, 0, 0, 0),
])
def test_cluster_sweeps_reproduce_colour_passes(L, R, c, schedule, or_mode, n_or):
    a, b = _pair(L, R, c, schedule, or_mode)
    T = np.geomspace(0.2, 2.0, R)
    acc_a = np.asarray(a.sweep(T, 1, n_or), float)
    acc_b = np.asarray(b.sweep(T, 1, n_or), float)
    assert np.all(np.abs(acc_b - acc_a) <= 1e-3 * np.maximum(acc_a, 1.0) + 1), (acc_a, acc_b)
    for r in range(R):
        _close_rounding(b.spins_f4(r), a.spins_f4(r))
    assert b.sweep_counter() == a.sweep_counter() == 1


def test_cluster_sweeps_then_per_pass_sweeps_continue_the_chain():
    a, b = _pair(8, 1, J3ON, 1, 0)
    a.sweep([0.5], 2, 1)
    b.sweep([0.5], 1, 1)
    b.set_cluster_sweeps(False)
    b.sweep([0.5], 1, 1)  # same sweep counter, so the same draws
    _close_rounding(b.spins_f4(0), a.spins_f4(0))
    assert b.sweep_counter() == a.sweep_counter() == 2


def test_cluster_sweeps_unsupported_cases():
    big = pc.pyrochlore_system(24, J1=1.0, J3=0.05)
    with pytest.raises(pc.PyroCMCError) as e:
        big.set_cluster_sweeps(True)
    assert e.value.code == _lib.ERR_UNSUPPORTED
    mixed = pc.pyrochlore_system([8, 12], J1=1.0, J3=0.05)
    with pytest.raises(pc.PyroCMCError):
        mixed.set_cluster_sweeps(True)
    lifted = pc.pyrochlore_system(8, J1=1.0, J3=0.05, update=1)
    with pytest.raises(pc.PyroCMCError):
        lifted.set_cluster_sweeps(True)
