"""pc_energy_noalloc: the energy entry point for callers that may not allocate
device memory (a program whose device memory belongs to a framework's caching
allocator, a loop that cannot take cudaFree's device-wide synchronisation). Its
partial sums live in a fixed array compiled into the library instead of a
buffer of the system.

Checked through the C ABI against the regular entry point (pc_energy) on two
calls in a row with different spins, so a stale scratch array from the first
call would show in the second; tolerance 1e-5 relative to the energy scale,
as in the other energy parity tests. This file is collected last; it also
runs on its own in a fresh process.
"""
import ctypes as C
import os
import subprocess
import sys

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


@pytest.mark.parametrize("L", [1, 2, 3, 8, 64])
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


def test_noalloc_rejects_misaligned_pointers():
    s = pc.pyrochlore_system(2, seed=4, **PARAMS)
    s.random_spins(3)
    out = torch.empty(8, dtype=torch.float64, device="cuda")
    with pytest.raises(pc.InvalidArgument, match="16-byte aligned"):
        _noalloc(s.spins_device_ptr(0) + 4, 2, out)
    p = np.zeros(7)
    rc = _lib.lib().pc_energy_noalloc(C.c_void_p(s.spins_device_ptr(0)), 2, p.ctypes.data_as(C.POINTER(C.c_double)),
                                      C.c_void_p(out.data_ptr() + 4), None)
    assert rc == 1 and b"8-byte aligned" in _lib.lib().pc_last_error()


_CHILD = r"""
import ctypes as C, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from pyro_cmc_b200 import _lib
lib = _lib.lib()
rt = C.CDLL("libcudart.so.12")
rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
rt.cudaFree.argtypes = [C.c_void_p]
L = 8
rng = np.random.default_rng(5)
v = rng.normal(size=(16 * L ** 3, 3))
v /= np.linalg.norm(v, axis=1, keepdims=True)
spins = np.zeros((16 * L ** 3, 4), np.float32)
spins[:, :3] = v
params = np.array([1.0, 0.1, -0.05, 0.7, 0.2, 0.1, -0.3])

def energy():
    d, o = C.c_void_p(), C.c_void_p()
    assert rt.cudaMalloc(C.byref(d), spins.nbytes) == 0 and rt.cudaMalloc(C.byref(o), 32) == 0
    assert rt.cudaMemcpy(d, spins.ctypes.data, spins.nbytes, 1) == 0
    rc = lib.pc_energy_noalloc(d, L, params.ctypes.data_as(C.POINTER(C.c_double)), o, None)
    assert rc == 0, lib.pc_last_error()
    assert rt.cudaDeviceSynchronize() == 0
    r = np.zeros(4)
    assert rt.cudaMemcpy(r.ctypes.data, o, 32, 2) == 0
    rt.cudaFree(d); rt.cudaFree(o)
    return r

r1 = energy()
assert rt.cudaDeviceReset() == 0
r2 = energy()
assert np.array_equal(r1, r2), (r1, r2)
print("same", r1[0])
"""


def test_noalloc_after_device_reset_in_fresh_process():
    """A process that resets its device (new primary context, the module and
    its array reloaded) gets the same result from its next call: the array's
    address is looked up again for the new context."""
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _CHILD, repo], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "same" in r.stdout
