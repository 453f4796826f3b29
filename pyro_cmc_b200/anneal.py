"""Run protocols of the reference drivers on the GPU engine.

generate_T_profile   include/cli_bits.hpp:250-289
anneal_batch         src/anneal.cpp:193-227, for K independent seeds at once
                     (the seeds become batched replicas of one system)
temper               src/temper.cpp:386-474 as batched on-device tempering
"""
from __future__ import annotations

import numpy as np

from .engine import pyrochlore_system


def generate_T_profile(T_hot: float, T_cold: float, T_sample, total_steps: int):
    """Log-spaced T_hot * f^i, i = 0..total_steps-1, f = (T_cold/T_hot)^(1/total_steps)
    (T_cold itself is not reached), merged in descending order with the
    T_sample values. Returns (T list, sorted list of the sample indices)."""
    factor = (T_cold / T_hot) ** (1.0 / total_steps)
    t = T_hot / factor
    sweep = []
    for _ in range(total_steps):
        t *= factor
        sweep.append(t)
    sweep.sort(reverse=True)
    samples = sorted(T_sample, reverse=True)
    T, idx = [], []
    i_sw = i_s = 0
    while i_sw < len(sweep) and i_s < len(samples):
        if sweep[i_sw] > samples[i_s]:
            T.append(sweep[i_sw])
            i_sw += 1
        else:
            idx.append(len(T))
            T.append(samples[i_s])
            i_s += 1
    for v in samples[i_s:]:
        idx.append(len(T))
        T.append(v)
    T.extend(sweep[i_sw:])
    return T, idx


def anneal_batch(K: int, L: int, J1: float, J2: float = 0.0, J3: float = 0.0, B=(0.0, 0.0, 0.0),
                 Delta: float = 1.0, T_hot: float = 10.0, T_cold: float | None = None, T_sample=(0.1,),
                 n_steps: int = 100, n_sweep: int = 16, n_burn_in: int = 16, n_sample: int = 64,
                 corr=("xx", "yy", "zz", "xy", "xz", "yz"), T_ref: float = 1.0, seed: int = 0,
                 init_seed: int | None = None, schedule: int = 0, update: int = 0, merge: bool = False):
    """The anneal protocol for K seeds at once: burn-in at T_hot, then for each
    T of the profile n_sweep sweeps and one energy sample; at the sample
    temperatures, n_sample x (n_sweep sweeps + one S(q) sample).
    Returns dict(T, sample_idx, e[K, n_T], ssf_sum/ssf_sq[K, n_Ts, n_corr, n_k, 2],
    n_ssf[n_Ts], accepted[K, n_T]); S(q) slots in visit (descending T) order.
    update 1: lifted Metropolis (src/anneal.cpp:184-188, --lifted).
    merge: also the seed merge of scripts/acc_runs.py over the K seeds,
    result["merged"] = dict(energy=..., ssf=[per T_sample dict]) with the S(q)
    part (sums, second moments, inter/intra-seed variances, spiral-plane
    invariants when the six correlators xx..yz are sampled) computed on the
    device (pc_ssf_merge)."""
    T_sample = list(T_sample)
    if T_cold is None:
        T_cold = min(T_sample)
    T_grid, S_idx = generate_T_profile(T_hot, T_cold, T_sample, n_steps)
    s = pyrochlore_system(L, J1=J1, J2=J2, J3=J3, Delta=Delta, B=B, T_ref=T_ref, seed=seed, n_replicas=K,
                          schedule=schedule, update=update)
    s.random_spins(seed if init_seed is None else init_seed)
    nTs = len(S_idx)
    s.ssf_configure(list(corr), max(1, K * nTs), [L] * max(1, K * nTs))
    e = np.zeros((K, len(T_grid)))
    acc = np.zeros((K, len(T_grid)), dtype=np.uint64)
    s.sweep(T_hot, n_burn_in, 1, count=False)
    slot = 0
    for i, T in enumerate(T_grid):
        acc[:, i] = s.sweep(T, n_sweep, 1)
        e[:, i], _ = s.energy()
        if i in S_idx:
            slots = np.arange(K, dtype=np.int32) + slot * K
            for _ in range(n_sample):
                s.sweep(T, n_sweep, 1, count=False)
                s.ssf_sample(slots)
            slot += 1
    nk = L ** 3
    merged = None
    if merge:
        six = {"xx", "yy", "zz", "xy", "xz", "yz"}.issubset(set(corr))
        e_cnt = np.ones_like(e)
        merged = dict(energy=dict(T_list=np.array(T_grid), E=e.sum(axis=0), E2=(e ** 2).sum(axis=0),
                                  n_samples=e_cnt.sum(axis=0), e_mean=e.mean(axis=0),
                                  e2_mean=(e ** 2).mean(axis=0), var=(e ** 2).mean(axis=0) - e.mean(axis=0) ** 2),
                      ssf=[s.ssf_merge(np.arange(K) + t * K, planes=six) for t in range(nTs)])
    ssum = np.zeros((K, nTs, len(corr), nk, 2))
    ssq = np.zeros_like(ssum)
    n_ssf = np.zeros(nTs, dtype=np.uint64)
    for t in range(nTs):
        for r in range(K):
            a, b, n = s.ssf_read(t * K + r)
            ssum[r, t] = a
            ssq[r, t] = b
            n_ssf[t] = n
    s.close()
    out = dict(T=np.array(T_grid), sample_idx=S_idx, e=e, ssf_sum=ssum, ssf_sq=ssq, n_ssf=n_ssf, accepted=acc)
    if merged is not None:
        out["merged"] = merged
    return out


def temper(L_list, T, J1: float, J2: float = 0.0, J3: float = 0.0, B=(0.0, 0.0, 0.0), Delta: float = 1.0,
           n_burn_in_rounds: int = 10, n_rounds: int = 100, n_sweep: int = 10, ssf_every: int = 0,
           corr=("xx", "yy", "zz"), seed: int = 0, schedule: int = 0):
    """Batched parallel tempering: replica r of size L_list[r] starts at T[r];
    replicas of equal L form one ladder. Returns per-slot (T, <e>, <e^2>,
    n samples), exchange statistics and the system (for SSF reads)."""
    s = pyrochlore_system(list(L_list), J1=J1, J2=J2, J3=J3, Delta=Delta, B=B, seed=seed, schedule=schedule)
    s.random_spins(seed)
    s.pt_configure(T)
    if ssf_every:
        s.ssf_configure(list(corr), len(L_list), sorted(L_list))
    s.pt_run(n_burn_in_rounds, n_sweep, 0)
    s.pt_reset_stats()
    s.pt_run(n_rounds, n_sweep, ssf_every)
    Ts, E, E2, n = s.pt_energy()
    att, acc = s.pt_exchange_stats()
    return dict(T=Ts, e=E / np.maximum(n, 1), e2=E2 / np.maximum(n, 1), n=n, attempts=att, accepts=acc, system=s)
