#!/usr/bin/env python3
"""Writes tests/golden/ref_mc_chains.npz from the reference's own Monte Carlo
code (src/MC.cpp compiled unchanged into oracle/_ref/libref_mc.so by
oracle/make_ref.sh; run that first, with the reference tree at hand).

The fixture lets the oracle be checked against the reference where the
reference cannot be built (e.g. a machine without the reference tree). For
each case it stores the start spins, the energy per cell, the local fields,
and after every one of a few sweeps (standard Metropolis + overrelaxation,
lifted u-form, lifted rotation form) the accepted count, the spins and the
lifting directions.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import ref  # noqa: E402

CASES = [
    # name, L, couplings, seed, T
    ("heis_L2", 2, dict(J1=1.0, J2=0.1, J3=0.05, Delta=1.0, B=(0.0, 0.0, 0.5)), 77, 0.5),
    ("xxz_L3", 3, dict(J1=-1.0, J2=0.3, J3=-0.02, Delta=0.6, B=(0.1, 0.2, 0.3)), 9, 0.3),
]
N_SWEEPS = 3


def start_spins(N, seed):
    rng = np.random.default_rng(seed)
    S = rng.normal(size=(N, 3))
    return S / np.linalg.norm(S, axis=1, keepdims=True)


def main():
    if not ref.available():
        sys.exit("oracle/_ref/libref_mc.so is missing: run oracle/make_ref.sh <reference tree> first")
    out = {}
    for name, L, c, seed, T in CASES:
        r = ref.RefSystem(L, seed=seed, **c)
        S0 = start_spins(r.N, seed)
        r.set_spins(S0)
        out[name + "/S0"] = S0
        out[name + "/energy"] = np.array(r.energy())
        out[name + "/field"] = r.local_fields()
        for mode in ("std", "u", "rot"):
            r = ref.RefSystem(L, seed=seed, **c)
            r.set_spins(S0)
            acc, spins, dirs = [], [], []
            for _ in range(N_SWEEPS):
                if mode == "std":
                    acc.append(r.sweep(T, 1, 1))
                else:
                    acc.append(r.sweep_lifted(T, 1, 1, rot=(mode == "rot")))
                spins.append(r.spins())
                dirs.append(r.lifted_dirs())
            out[f"{name}/{mode}/accepted"] = np.array(acc, np.int64)
            out[f"{name}/{mode}/spins"] = np.stack(spins)
            out[f"{name}/{mode}/dirs"] = np.stack(dirs)
    path = os.path.join(HERE, "ref_mc_chains.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main()
