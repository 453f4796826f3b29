"""Test infrastructure: the seed merge of scripts/acc_runs.py restated with
numpy, the checker of the device merge (pc_ssf_merge). Pinned against outputs
of the reference's own merge_group / plane_invariants
(tests/golden/acc_runs_merge.npz, made by tests/golden/make_merge_golden.py).
"""
from __future__ import annotations

import numpy as np


def merge_energy(E, E2, n):
    """acc_runs.py:291-298, 328-331 for per-seed energy sums E[K, n_T],
    E2[K, n_T], counts n[K, n_T]."""
    E_total, E2_total, n_total = E.sum(axis=0), E2.sum(axis=0), n.sum(axis=0)
    e_mean = E_total / n_total
    e2_mean = E2_total / n_total
    return dict(E=E_total, E2=E2_total, n_samples=n_total, e_mean=e_mean, e2_mean=e2_mean,
                var=e2_mean - e_mean ** 2)


def merge_ssf(static_corr, static_corr_2, n_samp):
    """acc_runs.py:301-354 for per-seed sums static_corr[K, ...], square sums
    static_corr_2[K, ...] (or None) with the sample count along axis 1 of the
    per-seed arrays given by n_samp[K, n_T] ([n_corr, n_T, n_k, 2] per seed)."""
    K = static_corr.shape[0]
    tot = static_corr.sum(axis=0)
    tot2 = (static_corr ** 2).sum(axis=0)
    n_tot = n_samp.sum(axis=0)
    n_ = (n_tot / K)[np.newaxis, :, np.newaxis, np.newaxis]
    out = dict(static_corr=tot, static_corr_2=tot2, n_samples=n_tot,
               var_inter=tot2 / (K * n_ ** 2) - (tot / (K * n_)) ** 2)
    if static_corr_2 is not None:
        out["var_intra"] = static_corr_2.sum(axis=0) / n_ - tot2 / n_ ** 2
    return out


def plane_invariants(static_corr, n_samp, labels):
    """acc_runs.py:103-167 for one seed: static_corr [n_corr, n_T, n_k, 2],
    n_samp [n_T]; returns w, chi_frac, tr [n_T, n_k] (None without the six
    correlators xx, yy, zz, xy, xz, yz)."""
    labels = [s.decode() if isinstance(s, bytes) else s for s in labels]
    need = ("xx", "yy", "zz", "xy", "xz", "yz")
    if not set(need).issubset(labels):
        return None
    idx = {l: i for i, l in enumerate(labels)}
    M = (static_corr[..., 0] + 1j * static_corr[..., 1]) / np.asarray(n_samp, float)[None, :, None]
    g = lambda l: M[idx[l]]
    Mxx, Myy, Mzz = g("xx").real, g("yy").real, g("zz").real
    Txy, Txz, Tyz = g("xy").real, g("xz").real, g("yz").real
    tr = Mxx + Myy + Mzz
    Txx, Tyy, Tzz = Mxx - tr / 3, Myy - tr / 3, Mzz - tr / 3
    I2 = Txx ** 2 + Tyy ** 2 + Tzz ** 2 + 2 * (Txy ** 2 + Txz ** 2 + Tyz ** 2)
    det = Txx * (Tyy * Tzz - Tyz ** 2) - Txy * (Txy * Tzz - Tyz * Txz) + Txz * (Txy * Tyz - Tyy * Txz)
    floor = 1e-6 * np.max(I2, axis=-1, keepdims=True) ** 1.5
    w = np.clip(3 * np.sqrt(6) * det / np.maximum(I2 ** 1.5, floor), -1, 1)
    kappa2 = 4 * (g("yz").imag ** 2 + g("xz").imag ** 2 + g("xy").imag ** 2)
    tr_floor = 1e-6 * np.max(tr, axis=-1, keepdims=True) + 1e-30
    chi = np.clip(np.sqrt(kappa2) / np.maximum(tr, tr_floor), 0, 1)
    return dict(w=w, chi_frac=chi, tr=tr)
