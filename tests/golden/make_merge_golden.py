"""Generates tests/golden/acc_runs_merge.npz: inputs and outputs of the
reference's own scripts/acc_runs.py (merge_group, plane_invariants) on small
synthetic seed files. Run in a container that has the reference checkout:

    python tests/golden/make_merge_golden.py <reference checkout>

acc_runs.py reads and writes HDF5 through h5py, which is not installed here; a
minimal in-memory stand-in for the calls it makes (File, Group, datasets,
attrs) is put in sys.modules before the import. The merge arithmetic is the
reference's, unmodified.
"""
import os
import sys
import types

import numpy as np

STORE = {}


class Group(dict):
    def __init__(self):
        super().__init__()
        self.attrs = {}

    def create_group(self, name):
        g = Group()
        self[name.strip("/")] = g
        return g

    def create_dataset(self, name, data):
        self[name.strip("/")] = np.array(data)


class File(Group):
    def __init__(self, name, mode="r"):
        super().__init__()
        self._name = name
        if mode == "r":
            self.update(STORE[name])
            self.attrs = STORE[name].attrs

    def __getitem__(self, key):
        node = self
        for part in key.strip("/").split("/"):
            node = dict.__getitem__(node, part)
        return node

    def __enter__(self):
        return self

    def __exit__(self, *a):
        g = Group()
        g.update(self)
        g.attrs = self.attrs
        STORE[self._name] = g


def seed_file(rng, name, K_idx, n_T=2, n_k=8, corr=("xx", "yy", "zz", "xy", "xz", "yz")):
    f = Group()
    e = f.create_group("energy")
    e.create_dataset("T_list", [0.5, 0.1])
    e.create_dataset("E", rng.normal(-10, 1, n_T))
    e.create_dataset("E2", rng.uniform(90, 110, n_T))
    e.create_dataset("n_samples", np.ones(n_T, dtype=np.uint64))
    g = f.create_group("geometry")
    g.create_dataset("index_cell", 16 * np.eye(3, dtype=np.int64))
    g.create_dataset("recip_vectors", np.eye(3) * 2 * np.pi / 16)
    s = f.create_group("ssf")
    s.create_dataset("T_list", [0.1, 0.5])
    s.create_dataset("corr_lookup", np.array([c.encode() for c in corr]))
    s.create_dataset("n_samples", np.array([4, 4], dtype=np.uint64))
    s.create_dataset("sl_positions", np.arange(48).reshape(16, 3))
    sc = rng.normal(0, 5, (len(corr), n_T, n_k, 2))
    sc[:3, ..., 0] = np.abs(sc[:3, ..., 0]) * 10  # diagonal correlators: positive real parts
    s.create_dataset("static_corr", sc)
    s.create_dataset("static_corr_2", sc ** 2 / 4 + rng.uniform(0, 50, sc.shape))
    s.attrs["n_spins"] = np.int32(128)
    s.attrs["k_dims"] = np.array([2, 2, 2], dtype=np.int32)
    STORE[name] = f
    return f


def main(ref):
    sys.modules["h5py"] = types.SimpleNamespace(File=File, Group=Group)
    sys.path.insert(0, os.path.join(ref, "scripts"))
    import acc_runs  # noqa: E402  (the reference's script)

    rng = np.random.default_rng(2024)
    names = [f"/virtual/run_L=2_J1=1_seed={s:x}_.out.h5" for s in (0xa1, 0xb2, 0xc3)]
    seeds = [seed_file(rng, n, i) for i, n in enumerate(names)]
    out = acc_runs.merge_group(names)
    m = STORE[out]
    pl = acc_runs.plane_invariants(seeds[0]["ssf"]["static_corr"], seeds[0]["ssf"]["n_samples"],
                                   seeds[0]["ssf"]["corr_lookup"])
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(
        os.path.join(here, "acc_runs_merge.npz"),
        in_E=np.stack([s["energy"]["E"] for s in seeds]), in_E2=np.stack([s["energy"]["E2"] for s in seeds]),
        in_n=np.stack([s["energy"]["n_samples"] for s in seeds]),
        in_sc=np.stack([s["ssf"]["static_corr"] for s in seeds]),
        in_sc2=np.stack([s["ssf"]["static_corr_2"] for s in seeds]),
        in_ssf_n=np.stack([s["ssf"]["n_samples"] for s in seeds]),
        corr=seeds[0]["ssf"]["corr_lookup"],
        out_E=m["energy"]["E"], out_E2=m["energy"]["E2"], out_n=m["energy"]["n_samples"],
        out_e_mean=m["energy"]["e_mean"], out_e2_mean=m["energy"]["e2_mean"], out_var=m["energy"]["var"],
        out_sc=m["ssf"]["static_corr"], out_sc2=m["ssf"]["static_corr_2"], out_ssf_n=m["ssf"]["n_samples"],
        out_var_inter=m["ssf"]["var_inter"], out_var_intra=m["ssf"]["var_intra"],
        pl_w=pl["w"], pl_chi=pl["chi_frac"], pl_tr=pl["tr"])
    print("wrote acc_runs_merge.npz from", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_merge_golden.py <reference tree>")
    main(sys.argv[1])
