"""The error path of the one device-side wait in the engine: the staged colour
pass (load variant 3) waits, with a bound, on the bulk copies of its neighbour
rows. With the bound of its first wait set to zero polls (pc_set_wait_limit)
every staged pass gives up at once: it sets the device error flag, waits for
its own copies at the full bound, skips its updates and the host call returns
PC_ERR_TIMEOUT. No GPU fault is involved: the copies complete, the kernels
return. The test checks the status, that nothing was updated, and that the
same system sweeps correctly (against the oracle's Philox mirror) once the
bound is restored."""
import numpy as np
import pytest

import oracle
import pyro_cmc_b200 as pc
from pyro_cmc_b200 import _lib

pytestmark = pytest.mark.gpu

C = dict(J1=1.0, J2=0.1, J3=0.05, Delta=1.0, B=(0.0, 0.0, 0.5))


@pytest.mark.parametrize("schedule", [0, 1])
def test_staged_pass_wait_runs_out_and_system_recovers(schedule):
    L, seed, T = 8, 77, 0.5
    g = pc.pyrochlore_system(L, seed=seed, schedule=schedule, **C)
    g.set_load_variant(3)
    assert g.load_variant() == 3
    g.random_spins(3)
    S0 = g.spins_f4().copy()
    g.set_wait_limit(0)
    with pytest.raises(pc.PyroCMCError) as ei:
        g.sweep(T, 1, 1)
    assert ei.value.code == _lib.ERR_TIMEOUT and "bounded wait" in str(ei.value)
    np.testing.assert_array_equal(g.spins_f4(), S0)  # every update of the sweep was skipped
    g.set_wait_limit(-1)
    o = oracle.System(L, seed=seed, **C)
    o.set_spins(g.spins())
    _, col = g.colours()
    sweep = g.sweep_counter()
    acc_g = int(g.sweep(T, 1, 1)[0])
    acc_o = int(o.sweep_philox(T, seed, 0, sweep, col, n_overrelax=1, or_mode=0, fused=bool(schedule)))
    assert abs(acc_g - acc_o) <= 2, (acc_g, acc_o)
    d = np.abs(g.spins() - o.spins()).max(axis=1)
    assert np.mean(d <= 1e-4) >= 0.999
    e, _ = g.energy()  # the device error flag was cleared: further calls succeed
    assert np.isfinite(e[0])
