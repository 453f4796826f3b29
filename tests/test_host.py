"""CPU tests of the product's host-side protocol code against the oracle."""
import numpy as np
import pytest

import oracle
from pyro_cmc_b200.anneal import generate_T_profile


@pytest.mark.parametrize("args", [(10.0, 0.05, [1.0, 0.1, 0.05], 100), (10.062, 0.02, [0.5, 0.1, 0.02], 200),
                                  (2.0, 0.01, [1.5, 1.0, 0.7, 0.5, 0.3, 0.1, 0.05, 0.01], 400),
                                  (1.0, 0.5, [0.7, 2.0], 5), (3.0, 0.1, [0.1], 1)])
def test_T_profile_matches_oracle(args):
    T, idx = generate_T_profile(*args)
    To, io = oracle.T_profile(*args)
    np.testing.assert_array_equal(np.array(T), To)
    assert list(idx) == list(io)


def _compile(tmp_path, name):
    import os
    import subprocess

    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    host = os.path.join(repo, "pyro_cmc_b200", "host")
    exe = tmp_path / name
    subprocess.run(["g++", "-O1", "-std=c++20", "-o", str(exe), os.path.join(repo, "tests", "cpp", name + ".cpp"),
                    os.path.join(host, "h5out.cpp"), os.path.join(host, "h5file.cpp")], check=True)
    return exe


@pytest.mark.parametrize("name", ["x.out.npz", "x.out.h5"])
def test_outfile_roundtrip(tmp_path, name):
    import subprocess

    from pyro_cmc_b200.h5compat import File

    exe = _compile(tmp_path, "outfile_roundtrip")
    out = tmp_path / name
    subprocess.run([str(exe), str(out)], check=True)
    with File(str(out)) as f:
        a = f["/ssf/static_corr"][:]
        assert a.shape == (2, 3, 4) and a.dtype == np.float64
        np.testing.assert_array_equal(a.ravel(), 0.5 * np.arange(24) - 3.0)
        assert (f["/geometry/index_cell"] == 8 * np.eye(3, dtype=np.int64)).all()
        assert f["/geometry/index_cell"].dtype == np.int64
        assert list(f["/energy/n_samples"]) == [7, 9] and f["/energy/n_samples"].dtype == np.uint64
        assert [s.decode() for s in f["/ssf/corr_lookup"]] == ["xx", "yz", "z"]
        assert int(f["/ssf"].attrs["n_spins"]) == 1024 and f["/ssf"].attrs["n_spins"].shape == ()
        assert list(f["/ssf"].attrs["k_dims"]) == [4, 4, 4] and f["/ssf"].attrs["k_dims"].dtype == np.int32
        assert set(f["/ssf"].keys()) == {"static_corr", "corr_lookup"}
        assert set(f.keys()) == {"ssf", "geometry", "energy"}
        assert "/ssf/static_corr" in f and "/ssf/nothing" not in f


@pytest.mark.parametrize("close", [True, False])
def test_hdf5_streaming_slices_survive_an_interrupted_run(tmp_path, close):
    """Slices written into reserved space are in the file as soon as they are
    written: a process that ends without closing leaves a readable file with
    the slices so far and zeros elsewhere (the reference's early-allocated
    /ssf/static_corr, include/ssf_manager.hpp:375-465)."""
    import subprocess

    from pyro_cmc_b200.h5compat import File

    exe = _compile(tmp_path, "h5_streaming")
    out = tmp_path / "s.out.h5"
    subprocess.run([str(exe), str(out), "close" if close else "kill"], check=True)
    want = np.zeros((2, 3, 4))
    for c in range(2):
        for t in (0, 2):
            want[c, t] = 100 * c + 10 * t + np.arange(4)
    with File(str(out)) as f:
        np.testing.assert_array_equal(f["/ssf/static_corr"][:], want)
        assert ("/ssf/T_list" in f) == close
        if close:
            np.testing.assert_array_equal(f["/ssf/T_list"][:], [0.1, 0.2, 0.3])


def test_hdf5_bytes_follow_the_published_format(tmp_path):
    """Byte-level checks of the writer against the HDF5 file format
    specification: lookup3 known answers, the version 2 superblock, the root
    group's link messages, the dataspace and datatype encodings and the global
    heap holding the variable-length strings."""
    import struct
    import subprocess

    from pyro_cmc_b200 import h5compat

    # lookup3 known answers (Jenkins' published test values)
    assert h5compat.lookup3(b"", 0) == 0xDEADBEEF
    assert h5compat.lookup3(b"Four score and seven years ago", 0) == 0x17770551
    assert h5compat.lookup3(b"Four score and seven years ago", 1) == 0xCD628161

    exe = _compile(tmp_path, "outfile_roundtrip")
    out = tmp_path / "b.out.h5"
    subprocess.run([str(exe), str(out)], check=True)
    raw = out.read_bytes()
    assert raw[:8] == b"\x89HDF\r\n\x1a\n"
    assert raw[8:12] == bytes([2, 8, 8, 0])
    base, ext, eof, root = struct.unpack_from("<4Q", raw, 12)
    assert base == 0 and ext == 0xFFFFFFFFFFFFFFFF and eof == len(raw)
    assert struct.unpack_from("<I", raw, 44)[0] == h5compat.lookup3(raw[:44])
    h5 = h5compat._H5(str(out))
    try:
        msgs = h5._messages(root)
        assert [t for t, _ in msgs] == [0x02, 0x0A, 0x06, 0x06, 0x06]
        ssf = h5.node(h5.node(root)["links"]["ssf"])
        sc = dict(h5._messages(ssf["links"]["static_corr"]))
        assert sc[0x01] == bytes([2, 3, 0, 1]) + struct.pack("<3Q", 2, 3, 4)
        assert sc[0x03] == bytes([0x11, 0x20, 63, 0]) + struct.pack("<IHHBBBBI", 8, 0, 64, 52, 11, 0, 52, 1023)
        ic = dict(h5._messages(h5.node(h5.node(root)["links"]["geometry"])["links"]["index_cell"]))
        assert ic[0x03] == bytes([0x10, 0x08, 0, 0]) + struct.pack("<IHH", 8, 0, 64)
        cl = dict(h5._messages(ssf["links"]["corr_lookup"]))
        assert cl[0x03] == bytes([0x19, 0x01, 0x01, 0]) + struct.pack("<I", 16) + \
            bytes([0x10, 0, 0, 0]) + struct.pack("<IHH", 1, 0, 8)
        lay = cl[0x08]
        addr = struct.unpack_from("<Q", lay, 2)[0]
        els = [struct.unpack_from("<IQI", raw, addr + 16 * i) for i in range(3)]
        assert [e[0] for e in els] == [2, 2, 1] and [e[2] for e in els] == [1, 2, 3]
        gcol = els[0][1]
        assert raw[gcol:gcol + 8] == b"GCOL" + bytes([1, 0, 0, 0])
        assert struct.unpack_from("<Q", raw, gcol + 8)[0] == 4096
        assert h5._heap(gcol) == {1: b"xx", 2: b"yz", 3: b"z"}
        # the free-space object (index 0) spans from its header to the end of the
        # collection, header included: 16 + 3 objects of 16 + 8 bytes before it
        free = gcol + 16 + 3 * 24
        idx, _ref, _r, fsize = struct.unpack_from("<HHIQ", raw, free)
        assert idx == 0 and fsize == 4096 - (free - gcol)
    finally:
        h5.close()


def test_anneal_dry_run_name_and_schedule():
    import os
    import subprocess

    from pyro_cmc_b200 import build

    build.build()
    exe = os.path.join(build.BIN, "anneal")
    out = subprocess.run([exe, "-o", "/tmp", "-s", "0xdeadbeef", "4", "--J1", "1", "--T_sample", "1.0", "0.1",
                          "0.05", "--dry_run"], check=True, capture_output=True, text=True).stdout.split("\n")
    # include/cli_bits.hpp:224-245 and src/anneal.cpp:156-161
    assert out[0] == "run_L=4_J1=1_J2=0_J3=0_Delta=1_B=0,0,0_seed=3735928559_Tc=0.05_sw=16_"
    rows = [r.split() for r in out[1:] if r.strip()]
    T = np.array([float(r[1]) for r in rows])
    To, io = oracle.T_profile(10.0, 0.05, [1.0, 0.1, 0.05], 100)
    np.testing.assert_array_equal(T, To)
    assert [int(r[0]) for r in rows if r[2] == "1"] == list(io)


def test_anneal_cli_errors():
    import os
    import subprocess

    from pyro_cmc_b200 import build

    build.build()
    exe = os.path.join(build.BIN, "anneal")
    r = subprocess.run([exe, "-o", "/tmp", "4", "--J1", "1", "--T_sample", "0.1"], capture_output=True, text=True)
    assert r.returncode == 1 and "--seed" in r.stderr
    r = subprocess.run([exe, "-o", "/tmp", "-s", "1", "4", "--J1", "1", "--J3", "0.1", "--Q", "0.5",
                        "--T_sample", "0.1", "--dry_run"], capture_output=True, text=True)
    assert r.returncode == 1 and "mutually exclusive" in r.stderr


def test_hdf5_edge_cases_and_corruption(tmp_path):
    """Empty and scalar datasets, an attribute on a dataset, implicit nested
    groups and a dataset added after a commit read back; a flipped byte in an
    object header is caught by its lookup3 checksum."""
    import subprocess

    from pyro_cmc_b200.h5compat import File

    exe = _compile(tmp_path, "h5_edges")
    out = tmp_path / "e.h5"
    subprocess.run([str(exe), str(out)], check=True)
    with File(str(out)) as f:
        assert list(f["/a/b/c/empty"]) == []
        np.testing.assert_array_equal(f["/a/b/vec"][:], [1.5, -2.0, 3.25, 0.0])
        assert float(f["/scalar"]) == 42.0 and f["/scalar"].shape == ()
        assert f["/a/none"].shape == (0,)
        np.testing.assert_array_equal(f["/a/b/c/late"][:], [-1, 1])
        assert set(f["/a/b"].keys()) == {"c", "vec"} and set(f["/a/b/c"].keys()) == {"empty", "late"}
        assert int(f._attrs("a/b/vec")["k"]) == 7
    raw = bytearray(out.read_bytes())
    i = raw.rfind(b"OHDR")
    raw[i + 12] ^= 0xFF
    bad = tmp_path / "bad.h5"
    bad.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="checksum"):
        with File(str(bad)) as f:
            f["/a/b/c/late"][:]



@pytest.mark.parametrize("split_J1", [True, False])
@pytest.mark.parametrize("Delta", [1.0, 0.6])
def test_parameter_gradient_mapping_on_torch_matches_numpy(split_J1, Delta):
    """The autograd energy's mapping from per-spec coupling gradients dE/dJ_spec
    (3x3) and dE/dB to dE/d[J1, J2, J3, Bx, By, Bz], formed with torch on the
    device (_param_grads_device), equals the numpy form (_param_grads) for the
    six XXZ J1 pair specs (Delta != 1 weights each by I + (Delta - 1) z_mu z_nu)
    and for the single isotropic J1 spec."""
    torch = pytest.importorskip("torch")
    from pyro_cmc_b200 import autograd as ag

    class _Sys:  # what the mapping reads of a System
        pass

    s = _Sys()
    s.pyro_params = dict(J1=1.0, J2=0.1, J3=-0.05, Delta=Delta, split_J1=split_J1)
    n_spec = (6 if split_J1 else 1) + 3
    rng = np.random.default_rng(3 + int(split_J1))
    gJ = rng.normal(size=(5, n_spec, 3, 3))
    gB = rng.normal(size=(5, 3))
    ref = ag._param_grads(s, gJ, gB)
    got = ag._param_grads_device(s, torch.as_tensor(gJ), torch.as_tensor(gB)).numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-13)
