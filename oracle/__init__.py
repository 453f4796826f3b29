"""The oracle: TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``oracle/liboracle.so``, an FP64 CPU restatement of the
reference pyro_cmc Monte Carlo path (src/MC.cpp, include/cli_bits.hpp,
include/ssf_manager.hpp, src/temper.cpp). Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (cpu_baseline leg and the
``--impl reference`` arm) may import this package, and only as the checker or
the CPU baseline. The product (``pyro_cmc_b200``) never imports it.

Parity status: pinned on the reference's own src/MC.cpp, compiled unchanged
into oracle/_ref/libref_mc.so (``oracle.ref``; tests/test_oracle_ref.py and the
fixture tests/golden/ref_mc_chains.npz), on the reference's geometry tables and
RNG header draws (tests/golden/), and on analytic known answers.
The lattice_lib conventions (DFT sign, flat-k order) are assumptions: parity
for the sign of Im S^{ab}(q) of off-diagonal correlators is unpinned.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_lib = None

_D = C.c_double
_I = C.c_int
_U64 = C.c_uint64
_U32 = C.c_uint32
_P = C.c_void_p
_DP = C.POINTER(C.c_double)
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
_U32P = C.POINTER(C.c_uint32)
_U64P = C.POINTER(C.c_uint64)


def build() -> None:
    """Compile liboracle.so (g++ -O3) if it is missing or older than its source."""
    src = os.path.join(_HERE, "pyro_oracle.cpp")
    if not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "liboracle.so"], check=True,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT)


def lib():
    global _lib
    if _lib is None:
        build()
        l = C.CDLL(_SO)
        l.orc_last_error.restype = C.c_char_p
        l.orc_create.restype = _P
        l.orc_create.argtypes = [_I, _D, _D, _D, _D, _DP, _D, _U64, _I]
        l.orc_destroy.argtypes = [_P]
        l.orc_num_spins.argtypes = [_P]
        l.orc_set_spins.argtypes = [_P, _DP]
        l.orc_get_spins.argtypes = [_P, _DP]
        l.orc_random_spins.argtypes = [_P, _U64]
        l.orc_reseed.argtypes = [_P, _U64]
        l.orc_set_field.argtypes = [_P, _DP]
        l.orc_positions.argtypes = [_P, _I64P, _I32P]
        l.orc_neighbours.argtypes = [_P, _I, _I, _I32P]
        l.orc_num_specs.argtypes = [_P]
        l.orc_spec_matrix.argtypes = [_P, _I, _DP]
        l.orc_spec_displacements.argtypes = [_P, _I, _I, _I64P, _I]
        l.orc_energy.restype = _D
        l.orc_energy.argtypes = [_P]
        l.orc_magnetisation.argtypes = [_P, _DP]
        l.orc_local_fields.argtypes = [_P, _DP]
        l.orc_coupling_grads.argtypes = [_P, _DP]
        l.orc_sweep.restype = _U64
        l.orc_sweep.argtypes = [_P, _D, _I, _I]
        l.orc_sweep_philox.restype = _U64
        l.orc_sweep_philox.argtypes = [_P, _D, _U64, _U32, _U64, _I, _I32P, _I, _I, _I]
        l.orc_sweep_lifted.restype = _U64
        l.orc_sweep_lifted.argtypes = [_P, _D, _I, _I, _I]
        l.orc_get_lifted.restype = None
        l.orc_get_lifted.argtypes = [_P, C.POINTER(C.c_int8)]
        l.orc_set_lifted.restype = None
        l.orc_set_lifted.argtypes = [_P, C.POINTER(C.c_int8)]
        l.orc_overrelax.argtypes = [_P, _DP, _I32P]
        l.orc_ssf.argtypes = [_P, _I32P, _I, _I, _DP, _DP]
        l.orc_T_profile.argtypes = [_D, _D, _DP, _I, _I, _DP, _I32P, _I]
        l.orc_anneal.argtypes = [_P, _D, _D, _DP, _I, _I, _I, _I, _I, _I32P, _I, _DP, _DP, _DP, _DP, _I]
        l.orc_temper.argtypes = [_I, _D, _D, _D, _D, _DP, _D, _U64, _DP, _I, _I, _I, _I, _I, _I, _DP, _DP, _U64P, _U64P]
        l.orc_bench_create.restype = _P
        l.orc_bench_create.argtypes = [_I, _D, _D, _D, _DP, _I, _U64]
        l.orc_bench_run.restype = _D
        l.orc_bench_run.argtypes = [_P, _D, _I]
        l.orc_bench_destroy.argtypes = [_P]
        l.orc_bench_sweeps.restype = _D
        l.orc_bench_sweeps.argtypes = [_I, _D, _D, _D, _DP, _D, _I, _I, _U64]
        l.orc_philox.argtypes = [_U32P, _U32P, _U32P]
        l.orc_xoshiro_draws.argtypes = [_U64, _I, _I, _DP, _U64P]
        _lib = l
    return _lib


def _dp(a):
    return a.ctypes.data_as(_DP)


def _arr(x, dtype):
    return np.ascontiguousarray(np.asarray(x, dtype=dtype))


CORR_AXES = {"x": 0, "y": 1, "z": 2}


def corr_pairs(names):
    """Correlator labels ("xx", "xy", ...) -> int32 [n,2] (ssf_manager.hpp:176-193)."""
    return np.array([[CORR_AXES[n[0]], CORR_AXES[n[1]]] for n in names], dtype=np.int32).reshape(-1, 2)


class System:
    """One reference-style lattice + MC_runner (FP64, sequential)."""

    def __init__(self, L, J1=1.0, J2=0.0, J3=0.0, Delta=1.0, B=(0, 0, 0), T_ref=1.0, seed=0, j1_mode=0):
        self.L = int(L)
        Bv = _arr(B, np.float64)
        self._h = lib().orc_create(self.L, J1, J2, J3, Delta, _dp(Bv), T_ref, seed, j1_mode)
        if not self._h:
            raise RuntimeError(lib().orc_last_error().decode())
        self.N = lib().orc_num_spins(self._h)
        self.Nc = self.L ** 3

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    # state
    def set_spins(self, S):
        S = _arr(S, np.float64).reshape(self.N, 3)
        lib().orc_set_spins(self._h, _dp(S))

    def spins(self):
        S = np.empty((self.N, 3))
        lib().orc_get_spins(self._h, _dp(S))
        return S

    def random_spins(self, seed):
        lib().orc_random_spins(self._h, seed)

    def reseed(self, seed):
        """Restart the runner's Xoroshiro stream from `seed` (a new chain on
        the same lattice, without rebuilding the bond shells)."""
        lib().orc_reseed(self._h, seed)

    def set_field(self, B):
        Bv = _arr(B, np.float64)
        lib().orc_set_field(self._h, _dp(Bv))

    def positions(self):
        pos = np.empty((self.N, 3), dtype=np.int64)
        sl = np.empty(self.N, dtype=np.int32)
        lib().orc_positions(self._h, pos.ctypes.data_as(_I64P), sl.ctypes.data_as(_I32P))
        return pos, sl

    def num_specs(self):
        return lib().orc_num_specs(self._h)

    def neighbours(self, spec, max_nb=16):
        out = np.empty((self.N, max_nb), dtype=np.int32)
        n = lib().orc_neighbours(self._h, spec, max_nb, out.ctypes.data_as(_I32P))
        if n < 0:
            raise ValueError("max_nb too small")
        return out[:, :n]

    def spec_matrix(self, spec):
        J = np.empty(9)
        lib().orc_spec_matrix(self._h, spec, _dp(J))
        return J.reshape(3, 3)

    def spec_displacements(self, spec, pyro_sl):
        out = np.empty((32, 3), dtype=np.int64)
        n = lib().orc_spec_displacements(self._h, spec, pyro_sl, out.ctypes.data_as(_I64P), 32)
        return out[:n]

    # observables
    def energy(self):
        return lib().orc_energy(self._h)

    def magnetisation(self):
        m = np.empty(3)
        lib().orc_magnetisation(self._h, _dp(m))
        return m

    def local_fields(self):
        h = np.empty((self.N, 3))
        lib().orc_local_fields(self._h, _dp(h))
        return h

    def coupling_grads(self):
        g = np.empty((self.num_specs(), 9))
        lib().orc_coupling_grads(self._h, _dp(g))
        return g.reshape(-1, 3, 3)

    # dynamics
    def sweep(self, T, n_sweeps=1, n_overrelax=1):
        return lib().orc_sweep(self._h, T, n_sweeps, n_overrelax)

    def sweep_philox(self, T, seed, replica, sweep, colour_of_sl, n_overrelax=1, or_mode=0, fused=False, update=0):
        """One sweep in the GPU's schedule with its Philox draws; update 0
        Metropolis, 1 lifted (u-form), 2 lifted (rotation form)."""
        col = _arr(colour_of_sl, np.int32)
        return lib().orc_sweep_philox(self._h, T, seed, replica, sweep, n_overrelax,
                                      col.ctypes.data_as(_I32P), or_mode, int(bool(fused)), int(update))

    def sweep_lifted(self, T, n_sweeps=1, n_overrelax=1, rot=False):
        """sweep_lifted_Metropolis(_rot) (src/MC.cpp:284-302) with the
        reference's Xoroshiro draws."""
        return lib().orc_sweep_lifted(self._h, T, n_sweeps, n_overrelax, int(bool(rot)))

    def lifted_dirs(self):
        d = np.empty(self.N, dtype=np.int8)
        lib().orc_get_lifted(self._h, d.ctypes.data_as(C.POINTER(C.c_int8)))
        return d

    def set_lifted_dirs(self, d):
        d = np.ascontiguousarray(np.asarray(d), dtype=np.int8)
        lib().orc_set_lifted(self._h, d.ctypes.data_as(C.POINTER(C.c_int8)))

    def overrelax(self, theta=None, colour_of_sl=None):
        col = None if colour_of_sl is None else _arr(colour_of_sl, np.int32)
        colp = None if col is None else col.ctypes.data_as(_I32P)
        if theta is None:
            lib().orc_overrelax(self._h, None, colp)
        else:
            th = _arr(theta, np.float64)
            lib().orc_overrelax(self._h, _dp(th), colp)

    def ssf(self, corr=("xx", "yy", "zz"), mode=0, resolved=False):
        cp = corr_pairs(corr)
        out = np.empty((len(cp), self.Nc, 2))
        res = np.empty((len(cp), self.Nc, 16, 16, 2)) if resolved else None
        lib().orc_ssf(self._h, cp.ctypes.data_as(_I32P), len(cp), mode, _dp(out),
                      _dp(res) if resolved else None)
        return (out, res) if resolved else out

    def anneal(self, T_hot, T_cold, T_sample, n_steps, n_sweep, n_burn_in, n_sample, corr=("xx", "yy", "zz")):
        ts = _arr(T_sample, np.float64)
        cp = corr_pairs(corr)
        maxT = n_steps + len(ts)
        T_out = np.empty(maxT)
        e_out = np.empty(maxT)
        ssum = np.zeros((len(ts), len(cp), self.Nc, 2))
        ssq = np.zeros_like(ssum)
        n = lib().orc_anneal(self._h, T_hot, T_cold, _dp(ts), len(ts), n_steps, n_sweep, n_burn_in, n_sample,
                             cp.ctypes.data_as(_I32P), len(cp), _dp(T_out), _dp(e_out), _dp(ssum), _dp(ssq), maxT)
        if n < 0:
            raise RuntimeError("anneal failed")
        return T_out[:n], e_out[:n], ssum, ssq


def T_profile(T_hot, T_cold, T_sample, total_steps):
    ts = _arr(T_sample, np.float64)
    maxn = total_steps + len(ts)
    T = np.empty(maxn)
    flag = np.empty(maxn, dtype=np.int32)
    n = lib().orc_T_profile(T_hot, T_cold, _dp(ts), len(ts), total_steps, _dp(T), flag.ctypes.data_as(_I32P), maxn)
    return T[:n], np.nonzero(flag[:n])[0]


def temper(L, T, J1=1.0, J2=0.0, J3=0.0, Delta=1.0, B=(0, 0, 0), T_ref=1.0, seed=0, n_burn_in=100,
           n_rounds=100, n_sweep=10, init_random=True, n_burn_rounds=0):
    """src/temper.cpp's tempering emulated in one process: n_burn_in sweeps
    per replica without exchanges, n_burn_rounds unmeasured rounds with
    exchanges, then n_rounds measured rounds. Returns per-slot sums of e and
    e^2 and the exchange attempts / accepts of each pair (slot, slot + 1)."""
    Tv = _arr(T, np.float64)
    R = len(Tv)
    Bv = _arr(B, np.float64)
    es = np.empty(R)
    e2 = np.empty(R)
    att = np.empty(R, dtype=np.uint64)
    acc = np.empty(R, dtype=np.uint64)
    rc = lib().orc_temper(L, J1, J2, J3, Delta, _dp(Bv), T_ref, seed, _dp(Tv), R, n_burn_in, n_burn_rounds, n_rounds,
                          n_sweep,
                          int(init_random), _dp(es), _dp(e2), att.ctypes.data_as(_U64P), acc.ctypes.data_as(_U64P))
    if rc:
        raise RuntimeError(lib().orc_last_error().decode())
    return es, e2, att, acc


class Bench:
    """n_threads independent reference-faithful lattices for CPU timing."""

    def __init__(self, L, J1, J2, J3, B, n_threads, seed=1):
        Bv = _arr(B, np.float64)
        self.n_threads = n_threads
        self.N = 16 * L ** 3
        self._h = lib().orc_bench_create(L, J1, J2, J3, _dp(Bv), n_threads, seed)

    def run(self, T, n_sweeps):
        """Aggregate spin-updates/s over all lattices for n_sweeps sweeps."""
        return lib().orc_bench_run(self._h, T, n_sweeps)

    def close(self):
        if self._h:
            lib().orc_bench_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def bench_sweeps(L, J1, J2, J3, B, T, n_sweeps, n_threads, seed=1):
    Bv = _arr(B, np.float64)
    return lib().orc_bench_sweeps(L, J1, J2, J3, _dp(Bv), T, n_sweeps, n_threads, seed)


def philox(ctr, key):
    c = _arr(ctr, np.uint32)
    k = _arr(key, np.uint32)
    out = np.empty(4, dtype=np.uint32)
    lib().orc_philox(c.ctypes.data_as(_U32P), k.ctypes.data_as(_U32P), out.ctypes.data_as(_U32P))
    return out


def xoshiro_draws(seed, kind, n):
    d = np.empty(n)
    u = np.empty(n, dtype=np.uint64)
    lib().orc_xoshiro_draws(seed, kind, n, _dp(d), u.ctypes.data_as(_U64P))
    return u if kind == 0 else d
