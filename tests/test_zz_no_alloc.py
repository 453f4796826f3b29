"""pc_energy_noalloc: the energy entry point for callers that may not allocate
device memory (a graph-capturing thread, a framework-owned memory pool, a loop
that cannot take cudaFree's device-wide synchronisation). Its partial sums live
in a fixed array compiled into the library instead of a buffer of the system.

Checked through the C ABI against the regular entry point (pc_energy) on two
calls in a row with different spins, so a stale scratch array from the first
call would show in the second; tolerance 1e-5 relative to the energy scale,
as in the other energy parity tests. This file is collected last; it also
runs on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import pyro_cmc_b200 as pc
from pyro_cmc_b200 import _lib

pytestmark = pytest.mark.gpu

PARAMS = dict(J1=1.0, J2=0.1, J3=-0.05, Delta=0.7, B=(0.2, 0.1, -0.3))


def _noalloc(spins_ptr, L, out):
    p = np.array([PARAMS["J1"], PARAMS["J2"], PARAMS["J3"], PARAMS["Delta"], *PARAMS["B"]], dtype=np.float64)
    rc = _lib.lib().pc_energy_noalloc(C.c_void_p(spins_ptr), L, p.ctypes.data_as(C.POINTER(C.c_double)),
                                      C.c_void_p(out.data_ptr()), None)
    _lib.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("L", [3, 8, 64])
def test_noalloc_energy_matches_regular_entry_point_twice(L):
    s = pc.pyrochlore_system(L, seed=4, **PARAMS)
    out = torch.empty(4, dtype=torch.float64, device="cuda")
    scale = 16 * (6 * 1.0 + 12 * 0.1 + 12 * 0.05 + 1)
    for call, seed in enumerate((11, 12)):
        s.random_spins(seed)
        e_ref, m_ref = s.energy()
        got = _noalloc(s.spins_device_ptr(0), L, out)
        assert abs(got[0] - e_ref[0]) <= 1e-5 * scale, (call, got[0], e_ref[0])
        np.testing.assert_allclose(got[1:], m_ref[0], rtol=0, atol=1e-6 * s.N())


def test_noalloc_rejects_lattices_beyond_its_scratch():
    out = torch.empty(4, dtype=torch.float64, device="cuda")
    with pytest.raises(pc.InvalidArgument, match="1..64"):
        _noalloc(out.data_ptr(), 65, out)
