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


def test_outfile_npz_roundtrip(tmp_path):
    import os
    import subprocess

    from pyro_cmc_b200.h5compat import File

    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "rt"
    subprocess.run(["g++", "-O1", "-std=c++20", "-o", str(exe), os.path.join(repo, "tests", "cpp", "outfile_roundtrip.cpp"),
                    os.path.join(repo, "pyro_cmc_b200", "host", "h5out.cpp")], check=True)
    out = tmp_path / "x.out.npz"
    subprocess.run([str(exe), str(out)], check=True)
    with File(str(out)) as f:
        a = f["/ssf/static_corr"][:]
        assert a.shape == (2, 3, 4) and a.dtype == np.float64
        np.testing.assert_array_equal(a.ravel(), 0.5 * np.arange(24) - 3.0)
        assert (f["/geometry/index_cell"] == 8 * np.eye(3, dtype=np.int64)).all()
        assert list(f["/energy/n_samples"]) == [7, 9] and f["/energy/n_samples"].dtype == np.uint64
        assert [s.decode() for s in f["/ssf/corr_lookup"]] == ["xx", "yz", "z"]
        assert int(f["/ssf"].attrs["n_spins"]) == 1024
        assert list(f["/ssf"].attrs["k_dims"]) == [4, 4, 4]
        assert set(f["/ssf"].keys()) == {"static_corr", "corr_lookup"}


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
