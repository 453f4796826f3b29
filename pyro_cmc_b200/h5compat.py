"""Reader for the drivers' output tree (<name>.out.npz, pyro_cmc_b200/host/h5out.hpp)
with the h5py-style access the reference's post-processing scripts use:

    f = File("run.out.npz")
    f["/ssf/static_corr"][:]        # dataset
    f["/ssf"].attrs["k_dims"]       # attribute
    list(f["/energy"].keys())
"""
from __future__ import annotations

import numpy as np


class Group:
    def __init__(self, f: "File", path: str):
        self._f = f
        self._path = path.strip("/")

    def _full(self, key: str) -> str:
        key = key.strip("/")
        return f"{self._path}/{key}" if self._path else key

    def __getitem__(self, key: str):
        return self._f[self._full(key)]

    def __contains__(self, key: str) -> bool:
        return self._full(key) in self._f

    def keys(self):
        pre = self._path + "/" if self._path else ""
        out = []
        for m in self._f._members:
            if m.startswith(pre):
                head = m[len(pre):].split("/")[0]
                if not head.startswith("@") and head not in out:
                    out.append(head)
        return out

    @property
    def attrs(self):
        pre = self._path + "/@" if self._path else "@"
        return {m[len(pre):]: self._f._z[m] for m in self._f._members if m.startswith(pre) and "/" not in m[len(pre):]}


class File(Group):
    def __init__(self, path: str, mode: str = "r"):
        if mode != "r":
            raise ValueError("read only")
        self._z = np.load(path)
        self._members = list(self._z.files)
        super().__init__(self, "")

    def __getitem__(self, key: str):
        key = key.strip("/")
        if key in self._members:
            return self._z[key]
        if any(m.startswith(key + "/") for m in self._members):
            return Group(self, key)
        raise KeyError(key)

    def __contains__(self, key: str) -> bool:
        key = key.strip("/")
        return key in self._members or any(m.startswith(key + "/") for m in self._members)

    def close(self):
        self._z.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
