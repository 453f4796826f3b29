"""Reader for the drivers' output trees with the h5py-style access the
reference's post-processing scripts use:

    f = File("run.out.h5")          # or "run.out.npz" (written with --npz)
    f["/ssf/static_corr"][:]        # dataset
    f["/ssf"].attrs["k_dims"]       # attribute
    list(f["/energy"].keys())

HDF5 files are read by a small parser of the format subset that
pyro_cmc_b200/host/h5file.hpp writes (and h5py reads): superblock version 2/3,
version 2 object headers (with continuation blocks), compact link storage,
contiguous or compact dataset layout, fixed-point, floating-point, fixed and
variable-length string datatypes, version 2/3 attribute messages. Metadata
checksums (Jenkins lookup3) are verified. Variable-length strings come back
as an object array of bytes, as h5py returns them.
"""
from __future__ import annotations

import mmap
import struct

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF


def lookup3(data: bytes, init: int = 0) -> int:
    """Jenkins' hashlittle (lookup3), the checksum of HDF5 metadata."""
    M = 0xFFFFFFFF

    def rot(x, k):
        return ((x << k) | (x >> (32 - k))) & M

    n = len(data)
    a = b = c = (0xDEADBEEF + n + init) & M
    k = 0
    while n > 12:
        a = (a + int.from_bytes(data[k:k + 4], "little")) & M
        b = (b + int.from_bytes(data[k + 4:k + 8], "little")) & M
        c = (c + int.from_bytes(data[k + 8:k + 12], "little")) & M
        a = (a - c) & M; a ^= rot(c, 4); c = (c + b) & M
        b = (b - a) & M; b ^= rot(a, 6); a = (a + c) & M
        c = (c - b) & M; c ^= rot(b, 8); b = (b + a) & M
        a = (a - c) & M; a ^= rot(c, 16); c = (c + b) & M
        b = (b - a) & M; b ^= rot(a, 19); a = (a + c) & M
        c = (c - b) & M; c ^= rot(b, 4); b = (b + a) & M
        n -= 12
        k += 12
    if n == 0:
        return c
    tail = data[k:k + n] + bytes(12 - n)
    a = (a + int.from_bytes(tail[0:4], "little")) & M
    b = (b + int.from_bytes(tail[4:8], "little")) & M
    c = (c + int.from_bytes(tail[8:12], "little")) & M
    c ^= b; c = (c - rot(b, 14)) & M
    a ^= c; a = (a - rot(c, 11)) & M
    b ^= a; b = (b - rot(a, 25)) & M
    c ^= b; c = (c - rot(b, 16)) & M
    a ^= c; a = (a - rot(c, 4)) & M
    b ^= a; b = (b - rot(a, 14)) & M
    c ^= b; c = (c - rot(b, 24)) & M
    return c


class _VLStr:
    """Marker datatype: variable-length string (16-byte elements)."""
    itemsize = 16


class _H5:
    """The object tree of an HDF5 file: path -> node dict."""

    def __init__(self, path: str):
        self._fh = open(path, "rb")
        self._m = mmap.mmap(self._fh.fileno(), 0, access=mmap.ACCESS_READ)
        m = self._m
        if m[:8] != _SIG:
            raise ValueError(f"{path}: not an HDF5 file")
        ver = m[8]
        if ver not in (2, 3):
            raise ValueError(f"{path}: superblock version {ver} is not supported")
        if m[9] != 8 or m[10] != 8:
            raise ValueError(f"{path}: only 8-byte offsets and lengths are supported")
        base, _ext, eof, root = struct.unpack_from("<4Q", m, 12)
        (ck,) = struct.unpack_from("<I", m, 44)
        if lookup3(m[:44]) != ck:
            raise ValueError(f"{path}: superblock checksum mismatch")
        if eof > len(m):
            raise ValueError(f"{path}: truncated (end of file {eof} > size {len(m)})")
        self._base = base
        self._heaps: dict[int, dict[int, bytes]] = {}
        self._nodes: dict[int, dict] = {}
        self.root = root

    def close(self):
        self._m.close()
        self._fh.close()

    # -- object headers ---------------------------------------------------
    def _messages(self, addr: int):
        m = self._m
        a = self._base + addr
        if m[a:a + 4] != b"OHDR" or m[a + 4] != 2:
            raise ValueError(f"object header at {addr}: only version 2 headers are supported")
        flags = m[a + 5]
        p = a + 6
        if flags & 0x20:
            p += 16
        if flags & 0x10:
            p += 4
        w = 1 << (flags & 3)
        size = int.from_bytes(m[p:p + w], "little")
        p += w
        blocks = [(a, p, p + size)]
        seen = set()
        out = []
        while blocks:
            start, p, end = blocks.pop(0)
            if start in seen:
                raise ValueError(f"object header at {addr}: continuation blocks form a cycle")
            seen.add(start)
            if end + 4 > len(m):
                raise ValueError(f"object header at {addr}: runs past the end of the file")
            (ck,) = struct.unpack_from("<I", m, end)
            if lookup3(m[start:end]) != ck:
                raise ValueError(f"object header at {start - self._base}: checksum mismatch")
            while end - p >= 4 + (2 if flags & 0x04 else 0):
                mtype = m[p]
                msize = int.from_bytes(m[p + 1:p + 3], "little")
                p += 4 + (2 if flags & 0x04 else 0)
                body = bytes(m[p:p + msize])
                p += msize
                if mtype == 0x10:  # continuation
                    caddr, clen = struct.unpack_from("<2Q", body, 0)
                    c = self._base + caddr
                    if m[c:c + 4] != b"OCHK":
                        raise ValueError("bad continuation block")
                    blocks.append((c, c + 4, c + clen - 4))
                else:
                    out.append((mtype, body))
        return out

    @staticmethod
    def _datatype(b: bytes, p: int = 0):
        cls, ver = b[p] & 0x0F, b[p] >> 4
        f0 = b[p + 1]
        (size,) = struct.unpack_from("<I", b, p + 4)
        if ver not in (1, 2, 3):
            raise ValueError(f"datatype version {ver}")
        if cls in (0, 1) and f0 & 1:
            raise ValueError("big-endian data is not supported")
        if cls == 0:
            return np.dtype(("<i" if f0 & 0x08 else "<u") + str(size))
        if cls == 1:
            return np.dtype("<f" + str(size))
        if cls == 3:
            return np.dtype("S" + str(size))
        if cls == 9 and (f0 & 0x0F) == 1:
            return _VLStr
        raise ValueError(f"datatype class {cls} is not supported")

    @staticmethod
    def _dataspace(b: bytes):
        ver, nd, fl = b[0], b[1], b[2]
        p = 4 if ver == 2 else 8
        if ver == 2 and b[3] == 0:
            return ()
        dims = struct.unpack_from(f"<{nd}Q", b, p)
        return tuple(int(d) for d in dims)

    def _heap(self, addr: int) -> dict[int, bytes]:
        h = self._heaps.get(addr)
        if h is not None:
            return h
        m = self._m
        a = self._base + addr
        if m[a:a + 4] != b"GCOL":
            raise ValueError(f"global heap at {addr}: bad signature")
        (csize,) = struct.unpack_from("<Q", m, a + 8)
        h = {}
        p, end = a + 16, a + csize
        while p + 16 <= end:
            idx, _ref, _r, osize = struct.unpack_from("<HHIQ", m, p)
            if idx == 0:
                break
            h[idx] = bytes(m[p + 16:p + 16 + osize])
            p += 16 + ((osize + 7) // 8) * 8
        self._heaps[addr] = h
        return h

    def _decode(self, raw: bytes | memoryview, dtype, shape):
        if dtype is _VLStr:
            n = int(np.prod(shape)) if shape else 1
            out = np.empty(n, dtype=object)
            for i in range(n):
                ln, caddr, idx = struct.unpack_from("<IQI", raw, 16 * i)
                out[i] = self._heap(caddr)[idx][:ln] if ln else b""
            return out.reshape(shape)
        return np.frombuffer(raw, dtype=dtype, count=int(np.prod(shape)) if shape else 1).reshape(shape).copy()

    def node(self, addr: int) -> dict:
        n = self._nodes.get(addr)
        if n is not None:
            return n
        n = {"links": {}, "attrs": {}, "dtype": None, "shape": None, "data": None}
        is_dataset = False
        layout = None
        for mtype, b in self._messages(addr):
            if mtype == 0x06:  # link
                fl = b[1]
                p = 2
                ltype = 0
                if fl & 0x08:
                    ltype = b[p]
                    p += 1
                if fl & 0x04:
                    p += 8
                if fl & 0x10:
                    p += 1
                w = 1 << (fl & 3)
                ln = int.from_bytes(b[p:p + w], "little")
                p += w
                name = b[p:p + ln].decode()
                p += ln
                if ltype == 0:
                    n["links"][name] = struct.unpack_from("<Q", b, p)[0]
            elif mtype == 0x01:
                n["shape"] = self._dataspace(b)
                is_dataset = True
            elif mtype == 0x03:
                n["dtype"] = self._datatype(b)
            elif mtype == 0x08:
                if b[0] != 3:
                    raise ValueError(f"layout version {b[0]} is not supported")
                if b[1] == 1:
                    layout = ("contiguous",) + struct.unpack_from("<2Q", b, 2)
                elif b[1] == 0:
                    (sz,) = struct.unpack_from("<H", b, 2)
                    layout = ("compact", b[4:4 + sz])
                else:
                    raise ValueError("chunked datasets are not supported")
            elif mtype == 0x0C:
                ver = b[0]
                nsz, tsz, ssz = struct.unpack_from("<3H", b, 2)
                p = 8 if ver == 2 else 9
                if ver not in (2, 3):
                    raise ValueError(f"attribute version {ver} is not supported")
                name = b[p:p + nsz].rstrip(b"\0").decode()
                p += nsz
                dt = self._datatype(b, p)
                p += tsz
                shape = self._dataspace(b[p:p + ssz])
                p += ssz
                n["attrs"][name] = self._decode(b[p:], dt, shape)
        if is_dataset:
            n["layout"] = layout
        self._nodes[addr] = n
        return n

    def resolve(self, path: str):
        n = self.node(self.root)
        for part in [q for q in path.split("/") if q]:
            a = n["links"].get(part)
            if a is None:
                return None
            n = self.node(a)
        return n

    def read(self, n: dict):
        lay = n["layout"]
        shape, dt = n["shape"], n["dtype"]
        count = int(np.prod(shape)) if shape else 1
        if lay is None:
            raise ValueError("dataset without a layout message")
        if lay[0] == "compact":
            raw = lay[1]
        else:
            _, addr, size = lay
            if addr == _UNDEF:
                raw = bytes(count * dt.itemsize)
            else:
                if size < count * dt.itemsize:
                    raise ValueError("dataset storage smaller than its dataspace")
                raw = memoryview(self._m)[self._base + addr:self._base + addr + count * dt.itemsize]
        try:
            return self._decode(raw, dt, shape)
        finally:
            if isinstance(raw, memoryview):
                raw.release()


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
        return self._f._keys(self._path)

    @property
    def attrs(self):
        return self._f._attrs(self._path)


class File(Group):
    def __init__(self, path: str, mode: str = "r"):
        if mode != "r":
            raise ValueError("read only")
        with open(path, "rb") as fh:
            sig = fh.read(8)
        self._h5 = _H5(path) if sig == _SIG else None
        if self._h5 is None:
            self._z = np.load(path)
            self._members = list(self._z.files)
        super().__init__(self, "")

    # -- HDF5 ---------------------------------------------------------------
    def _node(self, key: str):
        return self._h5.resolve(key)

    # -- common ---------------------------------------------------------------
    def __getitem__(self, key: str):
        key = key.strip("/")
        if self._h5 is not None:
            n = self._node(key)
            if n is None:
                raise KeyError(key)
            return Group(self, key) if n["shape"] is None else self._h5.read(n)
        if key in self._members:
            return self._z[key]
        if any(m.startswith(key + "/") for m in self._members):
            return Group(self, key)
        raise KeyError(key)

    def __contains__(self, key: str) -> bool:
        key = key.strip("/")
        if self._h5 is not None:
            return self._node(key) is not None
        return key in self._members or any(m.startswith(key + "/") for m in self._members)

    def _keys(self, path: str):
        if self._h5 is not None:
            n = self._node(path)
            return list(n["links"]) if n is not None else []
        pre = path + "/" if path else ""
        out = []
        for m in self._members:
            if m.startswith(pre):
                head = m[len(pre):].split("/")[0]
                if not head.startswith("@") and head not in out:
                    out.append(head)
        return out

    def _attrs(self, path: str):
        if self._h5 is not None:
            n = self._node(path)
            return dict(n["attrs"]) if n is not None else {}
        pre = path + "/@" if path else "@"
        return {m[len(pre):]: self._z[m] for m in self._members if m.startswith(pre) and "/" not in m[len(pre):]}

    def close(self):
        if self._h5 is not None:
            self._h5.close()
        else:
            self._z.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
