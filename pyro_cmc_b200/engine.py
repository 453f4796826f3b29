"""Python face of the engine: one `System` = a batch of pyrochlore replicas on
the GPU behind the C ABI (include/pyrocmc.h).

It mirrors the reference's MC_runner (include/MC.hpp:87-140) with batching:
`define_coupling` / `set_global_field` / `setup_lattice` / `sweep` /
`energy` / `local_field`, plus the ssf_manager and energy_manager roles
(`ssf_*`, `pt_*`). Arrays cross the boundary as numpy (host) or as device
addresses (torch tensors' data_ptr()).
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import call, lib

_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
_U64P = C.POINTER(C.c_uint64)


def _dp(a):
    return a.ctypes.data_as(_DP)


def _c(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


PAIRS = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))
LINK = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=np.int64)
FCC = np.array([[0, 0, 0], [0, 4, 4], [4, 0, 4], [4, 4, 0]], dtype=np.int64)


def displacements(kind: int, pyro_sl: int) -> np.ndarray:
    """Pyrochlore displacement table (see pc_pyrochlore_displacements):
    kind 1 J1, 2 J2, 3 J3a, 4 J3b, 10+nu J1 vectors landing on pyro_sl nu."""
    out = np.empty((64, 3), dtype=np.int64)
    n = C.c_int(0)
    call("pc_pyrochlore_displacements", kind, pyro_sl, out.ctypes.data_as(_I64P), 64, C.byref(n))
    return out[: n.value].copy()


def sublattice_offsets() -> np.ndarray:
    """r_sl = link[p] + R_fcc[f] for sl = 4f + p (pyrochlore_geometry.hpp:16-29)."""
    return np.array([LINK[sl % 4] + FCC[sl // 4] for sl in range(16)], dtype=np.int64)


def local_axis(p: int) -> np.ndarray:
    """Local [111] axis z_p = link[p]/sqrt(3) (pyrochlore::axis[p][2])."""
    return LINK[p].astype(np.float64) / np.sqrt(3.0)


class System:
    """A batch of replicas (L[r]^3 cubic cells each) on the current CUDA device."""

    def __init__(self, L: Sequence[int] | int, seed: int = 0, n_replicas: int | None = None):
        if np.isscalar(L):
            L = [int(L)] * (n_replicas or 1)
        self.L = [int(x) for x in L]
        self.R = len(self.L)
        self._N_total = sum(16 * x ** 3 for x in self.L)
        Lv = _c(self.L, np.int32)
        h = C.c_void_p()
        call("pc_create", self.R, Lv.ctypes.data_as(_I32P), C.c_uint64(seed & 0xFFFFFFFFFFFFFFFF), C.byref(h))
        self._h = h
        self.seed = seed
        self.spec_names: list[str] = []
        self.n_corr = 0
        self.corr_names: list[str] = []

    # ------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "_h", None):
            lib().pc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def Nc(self, r: int = 0) -> int:
        return self.L[r] ** 3

    def N(self, r: int = 0) -> int:
        return 16 * self.L[r] ** 3

    @property
    def N_total(self) -> int:
        return self._N_total

    def set_stream(self, stream_ptr: int):
        call("pc_set_stream", self._h, C.c_void_p(stream_ptr))
        self.stream_ptr = int(stream_ptr)

    # ----------------------------------------------------------- couplings
    def define_coupling(self, name: str, rel_vecs: Sequence[Sequence[Sequence[int]]], J):
        """MC_runner::define_coupling: rel_vecs[p] lists displacements from
        pyro_sl p; J (3x3) is applied by the lower-pyro_sl endpoint."""
        n = _c([len(rel_vecs[p]) for p in range(4)], np.int32)
        flat = [v for p in range(4) for v in rel_vecs[p]]
        rv = _c(np.array(flat, dtype=np.int64).reshape(-1, 3) if flat else np.zeros((0, 3)), np.int64)
        Jm = _c(np.asarray(J, dtype=np.float64).reshape(9), np.float64)
        call("pc_define_coupling", self._h, name.encode(), rv.ctypes.data_as(_I64P), n.ctypes.data_as(_I32P), _dp(Jm))
        self.spec_names.append(name)

    def define_pyrochlore(self, J1: float, J2: float = 0.0, J3: float = 0.0, Delta: float = 1.0,
                          split_J1: bool = True):
        """The coupling set of build_J1J2J3_h (include/cli_bits.hpp:175-200):
        J1 as six sublattice-pair XXZ specs J1[I + (Delta-1) z_mu (x) z_nu]
        (split_J1) or one isotropic spec on nn1_dist (test/spiral_byhand.cpp:81),
        then J2, J3a, J3b (defined even when zero)."""
        I3 = np.eye(3)
        self.pyro_params = dict(J1=J1, J2=J2, J3=J3, Delta=Delta, split_J1=split_J1)
        if split_J1:
            for mu, nu in PAIRS:
                rel = [[] for _ in range(4)]
                rel[mu] = displacements(10 + nu, mu).tolist()
                rel[nu] = displacements(10 + mu, nu).tolist()
                M = J1 * (I3 + (Delta - 1.0) * np.outer(local_axis(mu), local_axis(nu)))
                self.define_coupling(f"J1_{mu}{nu}", rel, M)
        else:
            self.define_coupling("J1", [displacements(1, p).tolist() for p in range(4)], J1 * I3)
        for name, kind, j in (("J2", 2, J2), ("J3a", 3, J3), ("J3b", 4, J3)):
            self.define_coupling(name, [displacements(kind, p).tolist() for p in range(4)], j * I3)

    def set_coupling_matrix(self, spec: int, J):
        Jm = _c(np.asarray(J, dtype=np.float64).reshape(9), np.float64)
        call("pc_set_coupling_matrix", self._h, int(spec), _dp(Jm))

    def set_coupling_matrices(self, specs: Sequence[int], Js):
        """Several coupling matrices at once (one rebuild of the tables; none
        when every matrix already holds its value)."""
        sp = _c(list(specs), np.int32)
        Jm = _c(np.asarray(Js, dtype=np.float64).reshape(len(sp), 9), np.float64)
        call("pc_set_coupling_matrices", self._h, len(sp), sp.ctypes.data_as(C.POINTER(C.c_int)), _dp(Jm))

    def set_global_field(self, B):
        Bv = _c(B, np.float64)
        call("pc_set_global_field", self._h, _dp(Bv))

    def get_global_field(self):
        B = np.empty(3)
        call("pc_get_global_field", self._h, _dp(B))
        return B

    def set_T_ref(self, T_ref: float):
        call("pc_set_T_ref", self._h, float(T_ref))

    def set_overrelax_mode(self, mode: int):
        call("pc_set_overrelax_mode", self._h, int(mode))

    def set_colouring(self, mode: int):
        """0: one colour class per sublattice in storage order (the
        reference's visiting order); 1: fewest classes."""
        call("pc_set_colouring", self._h, int(mode))

    def set_sweep_schedule(self, schedule: int):
        """0: the reference's order (Metropolis pass, then overrelaxation
        passes); 1: fused (Metropolis then overrelaxation per site in one
        colour pass, sharing the local field)."""
        call("pc_set_sweep_schedule", self._h, int(schedule))

    def set_update(self, mode: int):
        """0: Metropolis (sweep_local_Metropolis); 1: lifted Metropolis
        (sweep_lifted_Metropolis); 2: lifted, rotation form
        (sweep_lifted_Metropolis_rot). The lifting direction of each spin is
        the sign of its float4 w component."""
        call("pc_set_update", self._h, int(mode))

    def set_launch_overlap(self, on: bool):
        """Programmatic dependent launch between colour passes (default off)."""
        call("pc_set_launch_overlap", self._h, int(bool(on)))

    def set_cluster_sweeps(self, on: bool):
        """Cluster-resident sweeps for replicas of one size L <= 16 (one
        thread-block cluster per replica holds the lattice in distributed
        shared memory and runs all colour passes of a sweep call in one
        launch); raises PyroCMCError (code 4, unsupported) where the system
        does not qualify."""
        call("pc_set_cluster_sweeps", self._h, int(bool(on)))

    def cluster_sweeps(self) -> bool:
        v = C.c_int()
        call("pc_get_cluster_sweeps", self._h, C.byref(v))
        return bool(v.value)

    def set_pt_persistent(self, on: bool):
        """Tempering rounds (pt_run) in one persistent cooperative launch: all
        colour passes of all replicas, the energies and the exchanges, with
        grid barriers between the phases; raises PyroCMCError (code 4,
        unsupported) where the system does not qualify."""
        call("pc_set_pt_persistent", self._h, int(bool(on)))

    def pt_persistent(self) -> bool:
        v = C.c_int()
        call("pc_get_pt_persistent", self._h, C.byref(v))
        return bool(v.value)

    def set_kernel_path(self, force_generic: bool):
        """Force the generic bond-table kernels (True) or allow the structured
        pyrochlore kernels (False, default)."""
        call("pc_set_kernel_path", self._h, int(bool(force_generic)))

    def structured(self) -> bool:
        v = C.c_int(0)
        call("pc_kernel_path", self._h, C.byref(v))
        return bool(v.value)

    def setup_lattice(self):
        call("pc_setup_lattice", self._h)

    # ------------------------------------------------------------ inspection
    def colours(self):
        n = C.c_int(0)
        col = np.empty(16, dtype=np.int32)
        call("pc_colours", self._h, C.byref(n), col.ctypes.data_as(_I32P))
        return n.value, col

    def neighbour_table(self, spec: int, replica: int = 0, max_nb: int = 16):
        out = np.empty((self.N(replica), max_nb), dtype=np.int32)
        call("pc_neighbour_table", self._h, replica, spec, max_nb, out.ctypes.data_as(_I32P))
        return out

    def positions(self, replica: int = 0):
        pos = np.empty((self.N(replica), 3), dtype=np.int64)
        sl = np.empty(self.N(replica), dtype=np.int32)
        call("pc_site_positions", self._h, replica, pos.ctypes.data_as(_I64P), sl.ctypes.data_as(_I32P))
        return pos, sl

    def launch_count(self) -> int:
        n = C.c_uint64(0)
        call("pc_launch_count", self._h, C.byref(n))
        return n.value

    # ---------------------------------------------------------------- spins
    def set_spins(self, S, replica: int = 0):
        S = _c(S, np.float64).reshape(self.N(replica), 3)
        call("pc_set_spins", self._h, replica, _dp(S))

    def spins(self, replica: int = 0):
        S = np.empty((self.N(replica), 3))
        call("pc_get_spins", self._h, replica, _dp(S))
        return S

    def set_spins_f4(self, S4, replica: int = 0):
        S4 = _c(S4, np.float32).reshape(self.N(replica), 4)
        call("pc_set_spins_f4", self._h, replica, S4.ctypes.data_as(_FP))

    def spins_f4(self, replica: int = 0):
        S4 = np.empty((self.N(replica), 4), dtype=np.float32)
        call("pc_get_spins_f4", self._h, replica, S4.ctypes.data_as(_FP))
        return S4

    def random_spins(self, seed: int):
        call("pc_random_spins", self._h, C.c_uint64(seed))

    def spins_device_ptr(self, replica: int = 0) -> int:
        p = C.c_void_p()
        call("pc_spins_device", self._h, replica, C.byref(p))
        return p.value

    def sweep_counter(self) -> int:
        v = C.c_uint64(0)
        call("pc_get_sweep_counter", self._h, 0, C.byref(v))
        return v.value

    def set_sweep_counter(self, v: int):
        call("pc_set_sweep_counter", self._h, 0, C.c_uint64(v))

    # ------------------------------------------------------------------- MC
    def sweep(self, T, n_sweeps: int = 1, n_overrelax: int = 1, count: bool = True):
        """sweep_local_Metropolis(T, n_overrelax) n_sweeps times on every
        replica; returns accepted Metropolis moves per replica (count=False:
        returns None without waiting for the device)."""
        Tv = _c(np.broadcast_to(np.asarray(T, dtype=np.float64), (self.R,)), np.float64)
        if not count:
            call("pc_sweep", self._h, _dp(Tv), int(n_sweeps), int(n_overrelax), None)
            return None
        acc = np.zeros(self.R, dtype=np.uint64)
        call("pc_sweep", self._h, _dp(Tv), int(n_sweeps), int(n_overrelax), acc.ctypes.data_as(_U64P))
        return acc

    def overrelax_all(self):
        """One overrelaxation pass on every replica (Philox angles)."""
        call("pc_overrelax_all", self._h)

    def overrelax_theta(self, theta=None, replica: int = 0):
        if theta is None:
            call("pc_overrelax_theta", self._h, replica, None)
        else:
            th = _c(theta, np.float64)
            call("pc_overrelax_theta", self._h, replica, _dp(th))

    def energy(self):
        """Energy per cubic cell of every replica and the magnetisation sums."""
        e = np.empty(self.R)
        m = np.empty((self.R, 3))
        call("pc_energy", self._h, _dp(e), _dp(m))
        return e, m

    def local_field(self, replica: int = 0):
        h = np.empty((self.N(replica), 3))
        call("pc_local_field", self._h, replica, _dp(h))
        return h

    # ------------------------------------------------------------------ SSF
    ssf_resolved = False

    def ssf_set_resolved(self, on: bool):
        """Sublattice-resolved S(q) accumulators [n_corr][n_k][16][16][2]
        (call before ssf_configure)."""
        call("pc_ssf_set_resolved", self._h, int(bool(on)))
        self.ssf_resolved = bool(on)

    def _ssf_shape(self, nk: int):
        return (self.n_corr, nk, 16, 16, 2) if self.ssf_resolved else (self.n_corr, nk, 2)

    def ssf_configure(self, names: Sequence[str], n_slots: int, L_of_slot: Sequence[int] | None = None):
        arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
        if L_of_slot is None:
            L_of_slot = [self.L[0]] * n_slots
        Ls = _c(L_of_slot, np.int32)
        call("pc_ssf_configure", self._h, arr, len(names), int(n_slots), Ls.ctypes.data_as(_I32P))
        self._L_of_slot = [int(x) for x in L_of_slot]
        self.n_corr = len(names)
        self.corr_names = list(names)

    def ssf_sample(self, slot_of_replica):
        s = _c(np.broadcast_to(np.asarray(slot_of_replica), (self.R,)), np.int32)
        call("pc_ssf_sample", self._h, s.ctypes.data_as(_I32P))

    def ssf_read(self, slot: int, L: int | None = None):
        L = L or self.L[0]
        shape = self._ssf_shape(L ** 3)
        s = np.empty(shape)
        q = np.empty(shape)
        n = C.c_uint64(0)
        call("pc_ssf_read", self._h, slot, _dp(s), _dp(q), C.byref(n))
        return s, q, n.value

    def ssf_merge(self, slots, planes: bool = True):
        """Seed merge of the given slots on the device (scripts/acc_runs.py
        merge_group and plane_invariants): dict of static_corr,
        static_corr_2, var_inter, var_intra [n_corr, n_k, 2] and, with
        planes, w, chi_frac, tr [K, n_k]."""
        sl = _c(slots, np.int32)
        K = len(sl)
        nk = self.L_of_slot_hint(int(sl[0])) ** 3
        out = {k: np.empty((self.n_corr, nk, 2)) for k in ("static_corr", "static_corr_2", "var_inter", "var_intra")}
        if planes:
            out.update({k: np.empty((K, nk)) for k in ("w", "chi_frac", "tr")})
        P = lambda k: _dp(out[k]) if k in out else None
        call("pc_ssf_merge", self._h, sl.ctypes.data_as(_I32P), K, P("static_corr"), P("static_corr_2"),
             P("var_inter"), P("var_intra"), P("w"), P("chi_frac"), P("tr"))
        return out

    def L_of_slot_hint(self, slot: int) -> int:
        return self._L_of_slot[slot] if getattr(self, "_L_of_slot", None) else self.L[0]

    def ssf_clear(self, slot: int):
        call("pc_ssf_clear", self._h, slot)

    def ssf_current(self, replica: int = 0):
        out = np.empty(self._ssf_shape(self.Nc(replica)))
        call("pc_ssf_current", self._h, replica, _dp(out))
        return out

    def spin_ft(self, replica: int = 0):
        """save_ft_spin_state's array: the per-sublattice DFT over cells of
        each component, without sublattice phases, [3, 16, n_k, 2]
        (pc_spin_ft)."""
        out = np.empty((3, 16, self.Nc(replica), 2))
        call("pc_spin_ft", self._h, replica, _dp(out))
        return out

    def ssf_forward_device(self, out_ptr: int):
        call("pc_ssf_forward", self._h, C.c_void_p(out_ptr))

    def ssf_backward_device(self, grad_out_ptr: int, grad_spins_ptr: int):
        call("pc_ssf_backward", self._h, C.c_void_p(grad_out_ptr), C.c_void_p(grad_spins_ptr))

    def ssf_forward_keep(self, out_ptr: int) -> int:
        """pc_ssf_forward_keep: queued, keeps the amplitudes; returns their token."""
        t = C.c_uint64()
        call("pc_ssf_forward_keep", self._h, C.c_void_p(out_ptr), C.byref(t))
        return int(t.value)

    def ssf_backward_kept(self, token: int, grad_out_ptr: int, grad_spins_ptr: int):
        """pc_ssf_backward_kept: queued; reuses the amplitudes of `token` when
        still held."""
        call("pc_ssf_backward_kept", self._h, C.c_uint64(token), C.c_void_p(grad_out_ptr), C.c_void_p(grad_spins_ptr))

    # ----------------------------------------------------------- tempering
    def pt_configure(self, T):
        Tv = _c(T, np.float64)
        call("pc_pt_configure", self._h, _dp(Tv))

    def pt_run(self, n_rounds: int, n_sweep: int, ssf_every: int = 0):
        call("pc_pt_run", self._h, int(n_rounds), int(n_sweep), int(ssf_every))

    def pt_reset_stats(self):
        call("pc_pt_reset_stats", self._h)

    def pt_energy(self):
        T = np.empty(self.R)
        E = np.empty(self.R)
        E2 = np.empty(self.R)
        n = np.empty(self.R, dtype=np.uint64)
        call("pc_pt_read_energy", self._h, _dp(T), _dp(E), _dp(E2), n.ctypes.data_as(_U64P))
        return T, E, E2, n

    def pt_exchange_stats(self):
        a = np.empty(self.R, dtype=np.uint64)
        b = np.empty(self.R, dtype=np.uint64)
        call("pc_pt_read_exchange", self._h, a.ctypes.data_as(_U64P), b.ctypes.data_as(_U64P))
        return a, b

    def pt_slots(self):
        s = np.empty(self.R, dtype=np.int32)
        call("pc_pt_slots", self._h, s.ctypes.data_as(_I32P))
        return s

    # -------------------------------------------------------- gradients
    def energy_grad(self, g=None, grad_spins_ptr: int | None = None, couplings: bool = True):
        """Energy per cell, dE/dJ_spec (per replica, per spec, 3x3; None with
        couplings=False, which skips forming them) and dE/dB, scaled by
        upstream g[r]; writes dE/dS into grad_spins_ptr if given."""
        n_spec = len(self.spec_names)
        e = np.empty(self.R)
        gJ = np.empty((self.R, n_spec, 9)) if couplings else None
        gB = np.empty((self.R, 3))
        gv = None if g is None else _c(np.broadcast_to(np.asarray(g, dtype=np.float64), (self.R,)), np.float64)
        call("pc_energy_grad", self._h, None if gv is None else _dp(gv), _dp(e),
             None if grad_spins_ptr is None else C.c_void_p(grad_spins_ptr), None if gJ is None else _dp(gJ),
             _dp(gB))
        return e, None if gJ is None else gJ.reshape(self.R, n_spec, 3, 3), gB

    def energy_device(self, e_ptr: int):
        """Queues the energy per cell of every replica into the device array
        at e_ptr (R doubles) on the system's stream, without waiting."""
        call("pc_energy_device", self._h, C.c_void_p(e_ptr))

    def energy_groups_device(self, e_ptr: int, out_ptr: int):
        """pc_energy_groups_device: energies (R device doubles) and per replica
        [the six coupling groups' bare bond sums, sum S] (R x 9 device
        doubles), queued; raises PyroCMCError code 4 (unsupported) unless the
        couplings are isotropic, nonzero and uniform over the sublattices."""
        call("pc_energy_groups_device", self._h, C.c_void_p(e_ptr), C.c_void_p(out_ptr))

    def energy_grad_device(self, g_ptr: int | None, grad_spins_ptr: int | None, sums_ptr: int | None,
                           couplings: bool):
        """Queues pc_energy_grad_device: upstream g (R device doubles, None:
        1), dE/dS into grad_spins_ptr, per-replica sums (R x (4 + 9 n_spec)
        device doubles) into sums_ptr; returns without waiting."""
        call("pc_energy_grad_device", self._h, None if g_ptr is None else C.c_void_p(g_ptr),
             None if grad_spins_ptr is None else C.c_void_p(grad_spins_ptr),
             None if sums_ptr is None else C.c_void_p(sums_ptr), int(bool(couplings)))

    def energy_grad_field(self, field_ptr: int, g=None, grad_ptr: int | None = None, couplings: bool = True):
        """energy_grad evaluated on the device field at field_ptr (float4
        [N_total]) instead of the system's spins (pc_energy_grad_field)."""
        n_spec = len(self.spec_names)
        e = np.empty(self.R)
        gJ = np.empty((self.R, n_spec, 9)) if couplings else None
        gB = np.empty((self.R, 3))
        gv = None if g is None else _c(np.broadcast_to(np.asarray(g, dtype=np.float64), (self.R,)), np.float64)
        call("pc_energy_grad_field", self._h, C.c_void_p(field_ptr), None if gv is None else _dp(gv), _dp(e),
             None if grad_ptr is None else C.c_void_p(grad_ptr), None if gJ is None else _dp(gJ), _dp(gB))
        return e, None if gJ is None else gJ.reshape(self.R, n_spec, 3, 3), gB

    # ---------------------------------------------------------------- tuning
    def autotune(self):
        """Picks the fastest tile shape and neighbour-load variant by timing
        sweeps on this system; returns (threads, ctas_per_sm, load_variant)."""
        call("pc_autotune", self._h)
        return (*self.tile(), self.load_variant())

    def load_variant(self) -> int:
        v = C.c_int(0)
        call("pc_get_load_variant", self._h, C.byref(v))
        return v.value

    def set_load_variant(self, v: int):
        call("pc_set_load_variant", self._h, int(v))

    def tile(self):
        t = C.c_int(0)
        c = C.c_int(0)
        call("pc_get_tile", self._h, C.byref(t), C.byref(c))
        return t.value, c.value

    def set_tile(self, threads: int, ctas_per_sm: int):
        call("pc_set_tile", self._h, threads, ctas_per_sm)

    def set_wait_limit(self, polls: int):
        """Bound of the staged colour pass's first wait on its copies
        (pc_set_wait_limit; < 0 restores the default)."""
        call("pc_set_wait_limit", self._h, int(polls))

    def set_kernel_timing(self, on: bool):
        call("pc_set_kernel_timing", self._h, int(bool(on)))

    def kernel_times(self):
        a = C.c_double(0)
        b = C.c_double(0)
        call("pc_last_kernel_times", self._h, C.byref(a), C.byref(b))
        return a.value, b.value

    def step_host(self, S4_in, S4_out, T: float, n_sweep: int, ssf_every: int = 0, ssf_slot: int = -1):
        """One host-buffer step (pc_step_host): upload spins, n_sweep sweeps
        with an SSF sample every ssf_every sweeps, one energy sample, download.
        S4_in / S4_out: float32 [N, 4] numpy arrays (pinned for full speed)."""
        e = C.c_double(0)
        acc = C.c_uint64(0)
        call("pc_step_host", self._h, S4_in.ctypes.data_as(_FP), S4_out.ctypes.data_as(_FP), float(T),
             int(n_sweep), int(ssf_every), int(ssf_slot), C.byref(e), C.byref(acc))
        return e.value, acc.value

    def step_host3(self, S3_in, S3_out, T: float, n_sweep: int, ssf_every: int = 0, ssf_slot: int = -1):
        """step_host with packed host spins (pc_step_host3): float32 [N, 3]
        numpy arrays (pinned for full speed), 12 bytes a spin over the bus;
        the lifting directions stay on the device."""
        for a in (S3_in, S3_out):
            if a.dtype != np.float32 or a.shape != (self.N(0), 3) or not a.flags["C_CONTIGUOUS"]:
                raise ValueError("step_host3 takes C-contiguous float32 [N, 3] arrays")
        e = C.c_double(0)
        acc = C.c_uint64(0)
        call("pc_step_host3", self._h, S3_in.ctypes.data_as(_FP), S3_out.ctypes.data_as(_FP), float(T),
             int(n_sweep), int(ssf_every), int(ssf_slot), C.byref(e), C.byref(acc))
        return e.value, acc.value


def pyrochlore_system(L, J1=1.0, J2=0.0, J3=0.0, Delta=1.0, B=(0.0, 0.0, 0.0), T_ref=1.0, seed=0,
                      n_replicas=None, split_J1=True, overrelax_mode=0, colouring=0, generic=False,
                      schedule=0, update=0) -> System:
    """build_J1J2J3_h (include/cli_bits.hpp:144-207) on the GPU engine."""
    s = System(L, seed=seed, n_replicas=n_replicas)
    s.set_colouring(colouring)
    s.set_kernel_path(generic)
    s.set_sweep_schedule(schedule)
    s.set_update(update)
    s.define_pyrochlore(J1, J2, J3, Delta, split_J1=split_J1)
    s.set_global_field(B)
    s.set_T_ref(T_ref)
    s.set_overrelax_mode(overrelax_mode)
    s.setup_lattice()
    return s
