"""The reference's own Monte Carlo code, compiled: TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``oracle/_ref/libref_mc.so``, which ``oracle/make_ref.sh``
builds from the reference's unchanged ``src/MC.cpp`` (plus
``oracle/ref_mc_main.cpp`` and the lattice_lib / HDF5 stand-ins in
``oracle/ref_shim/``). The tests use it to pin the oracle's restatement
(``oracle/pyro_oracle.cpp``) on the reference itself; ``bench.py`` may time its
sweep as the reference's CPU baseline. The product never loads it.

``available()`` is False where the library was not built (the reference tree
is needed to build it); callers skip then.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(_HERE, "_ref", "libref_mc.so")
_lib = None

_D, _I, _U64, _P = C.c_double, C.c_int, C.c_uint64, C.c_void_p
_DP = C.POINTER(C.c_double)
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)


def available() -> bool:
    return os.path.exists(SO)


def lib():
    global _lib
    if _lib is None:
        l = C.CDLL(SO)
        l.ref_last_error.restype = C.c_char_p
        l.ref_create.restype = _P
        l.ref_create.argtypes = [_I, _D, _D, _D, _D, _DP, _D, _U64]
        l.ref_destroy.argtypes = [_P]
        l.ref_num_spins.restype = C.c_int64
        l.ref_num_spins.argtypes = [_P]
        l.ref_set_spins.argtypes = [_P, _DP]
        l.ref_get_spins.argtypes = [_P, _DP]
        l.ref_positions.argtypes = [_P, _I64P]
        l.ref_shells.restype = C.c_int64
        l.ref_shells.argtypes = [_P, _I32P, _DP, C.c_int64, _I32P, C.c_int64]
        l.ref_energy.restype = _D
        l.ref_energy.argtypes = [_P]
        l.ref_local_fields.argtypes = [_P, _DP]
        l.ref_sweep.restype = _U64
        l.ref_sweep.argtypes = [_P, _D, _I, _I]
        l.ref_sweep_lifted.restype = _U64
        l.ref_sweep_lifted.argtypes = [_P, _D, _I, _I, _I]
        l.ref_overrelax_all.argtypes = [_P]
        l.ref_get_lifted.argtypes = [_P, C.POINTER(C.c_int8)]
        _lib = l
    return _lib


class RefSystem:
    """One reference Lattice + MC_runner (src/MC.cpp, compiled unchanged) with
    build_J1J2J3_h's couplings, constructed with the raw seed."""

    def __init__(self, L, J1=1.0, J2=0.0, J3=0.0, Delta=1.0, B=(0, 0, 0), T_ref=1.0, seed=0):
        self.L = int(L)
        Bv = np.ascontiguousarray(B, dtype=np.float64)
        self._h = lib().ref_create(self.L, J1, J2, J3, Delta, Bv.ctypes.data_as(_DP), T_ref, seed)
        if not self._h:
            raise RuntimeError(lib().ref_last_error().decode())
        self.N = int(lib().ref_num_spins(self._h))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ref_destroy(self._h)
            self._h = None

    def set_spins(self, S):
        S = np.ascontiguousarray(S, dtype=np.float64).reshape(self.N, 3)
        lib().ref_set_spins(self._h, S.ctypes.data_as(_DP))

    def spins(self):
        S = np.zeros((self.N, 3))
        lib().ref_get_spins(self._h, S.ctypes.data_as(_DP))
        return S

    def positions(self):
        p = np.zeros((self.N, 3), np.int64)
        lib().ref_positions(self._h, p.ctypes.data_as(_I64P))
        return p

    def shells(self):
        """Per site: list of (3x3 matrix, neighbour site indices) in setup order."""
        n_sh = np.zeros(self.N, np.int32)
        max_m = self.N * 16
        mats = np.zeros((max_m, 9))
        idx = np.zeros(self.N * 64, np.int32)
        w = lib().ref_shells(self._h, n_sh.ctypes.data_as(_I32P), mats.ctypes.data_as(_DP), max_m,
                             idx.ctypes.data_as(_I32P), idx.size)
        if w < 0:
            raise RuntimeError("shell buffer too small")
        out, m, p = [], 0, 0
        for i in range(self.N):
            site = []
            for _ in range(int(n_sh[i])):
                n = int(idx[p])
                site.append((mats[m].reshape(3, 3).copy(), idx[p + 1:p + 1 + n].copy()))
                p += 1 + n
                m += 1
            out.append(site)
        return out

    def energy(self):
        return float(lib().ref_energy(self._h))

    def local_fields(self):
        h = np.zeros((self.N, 3))
        lib().ref_local_fields(self._h, h.ctypes.data_as(_DP))
        return h

    def sweep(self, T, n_sweeps=1, n_overrelax=1):
        return int(lib().ref_sweep(self._h, T, n_sweeps, n_overrelax))

    def sweep_lifted(self, T, n_sweeps=1, n_overrelax=1, rot=False):
        return int(lib().ref_sweep_lifted(self._h, T, n_sweeps, n_overrelax, 1 if rot else 0))

    def overrelax_all(self):
        lib().ref_overrelax_all(self._h)

    def lifted_dirs(self):
        d = np.zeros(self.N, np.int8)
        lib().ref_get_lifted(self._h, d.ctypes.data_as(C.POINTER(C.c_int8)))
        return d
