"""The C++ drivers (anneal, fieldcool, temper, spiral_byhand) end to end on the
GPU: output tree, schedule, and agreement with the Python protocol and the
oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import pyro_cmc_b200 as pc
from pyro_cmc_b200 import build
from pyro_cmc_b200.anneal import anneal_batch, generate_T_profile
from pyro_cmc_b200.h5compat import File

pytestmark = pytest.mark.gpu


def run(exe, *args, cwd=None):
    build.build()
    r = subprocess.run([os.path.join(build.BIN, exe), *map(str, args)], capture_output=True, text=True, cwd=cwd)
    assert r.returncode == 0, r.stderr + r.stdout
    return r.stdout


def only(tmp_path, suffix):
    files = [f for f in os.listdir(tmp_path) if f.endswith(suffix)]
    assert len(files) == 1, files
    return os.path.join(tmp_path, files[0])


def test_anneal_driver_output_and_determinism(tmp_path):
    args = ["-o", tmp_path, "-s", 77, 2, "--J1", 1, "--J2", -0.1, "--J3", 0.05, "--T_sample", 1.0, 0.5,
            "--n_steps", 10, "--n_sweep", 4, "--n_burn_in", 4, "--n_sample", 4, "--init_uniform",
            "--correlators", "xx", "yy", "zz", "xy", "xz", "yz", "yx", "zx", "zy", "--save_state"]
    out = run("anneal", *args)
    assert "[anneal] Iter" in out and "Saved to" in out
    path = only(tmp_path, ".out.h5")
    T_grid, S_idx = generate_T_profile(10.0, 0.5, [1.0, 0.5], 10)
    with File(path) as f:
        np.testing.assert_array_equal(f["/energy/T_list"], T_grid)
        E = f["/energy/E"][:]
        assert np.isfinite(E).all() and (f["/energy/n_samples"][:] == 1).all()
        sc = f["/ssf/static_corr"][:]
        assert sc.shape == (9, 2, 8, 2)
        np.testing.assert_array_equal(f["/ssf/T_list"], [0.5, 1.0])
        assert list(f["/ssf/n_samples"]) == [4, 4]
        assert [s.decode() for s in f["/ssf/corr_lookup"]][:3] == ["xx", "yy", "zz"]
        assert (sc[:3, ..., 0] >= -1e-6).all()
        assert int(f["/ssf"].attrs["n_spins"]) == 128 and list(f["/ssf"].attrs["k_dims"]) == [2, 2, 2]
        assert (f["/geometry/index_cell"] == 16 * np.eye(3)).all()
        assert f["/ssf/sl_positions"].shape == (16, 3)
    with File(only(tmp_path, ".spins.h5")) as f:
        assert f["/spin_orientation"].shape == (128, 3) and f["/spin_pos"].dtype == np.int32
        assert np.allclose(np.linalg.norm(f["/spin_orientation"], axis=1), 1.0, atol=1e-5)
    # the same run through the Python protocol: identical calls, identical chain
    py = anneal_batch(K=1, L=2, J1=1, J2=-0.1, J3=0.05, T_hot=10.0, T_sample=[1.0, 0.5], n_steps=10, n_sweep=4,
                      n_burn_in=4, n_sample=4, corr=["xx"], seed=77, init_seed=77 ^ 0x5EED)
    np.testing.assert_array_equal(py["e"][0], E)


def test_spiral_byhand_driver(tmp_path):
    out = run("spiral_byhand", "-o", tmp_path, 4, 1, 2, 0)
    E = float(out.split("Total E = ")[1].split()[0])
    o = oracle.System(4, J1=-1.0, j1_mode=1)
    with File(only(tmp_path, ".spins.h5")) as f:
        o.set_spins(f["/spin_orientation"][:].astype(np.float32).astype(np.float64))
    assert E == pytest.approx(o.energy(), abs=1e-4)
    with File(only(tmp_path, ".out.h5")) as f:
        sc = f["/ssf/static_corr"][:]
        tot = sc[1, 0, :, 0] + sc[2, 0, :, 0]
        N = 16 * 64
        assert tot[(1 * 4 + 2) * 4 + 0] == pytest.approx(N * N / 2, rel=1e-5)


def test_temper_driver(tmp_path):
    out = run("temper", "-o", tmp_path, "-s", 5, "--n_replicas", 6, 2, "--J1", 1, "--J3", 0.02, "-B", 0, 0, 0.1,
              "--T_hot", 2.0, "--T_sample", 0.5, "--n_sweep", 4, "--n_burn_in", 8, "--n_sample", 20, "--init_uniform",
              "--save_state")
    assert "per-pair swap acceptance" in out
    with File(only(tmp_path, ".out.h5")) as f:
        T = f["/energy/T_list"][:]
        assert len(T) == 6 and (np.diff(T) > 0).all()
        assert (f["/energy/n_samples"][:] == 20).all()
        assert np.isfinite(f["/energy/E"][:]).all()
        np.testing.assert_array_equal(f["/ssf/T_list"], [0.5])
        assert f["/ssf/static_corr"].shape == (3, 1, 8, 2)
        assert list(f["/ssf/n_samples"]) == [20]


def test_fieldcool_driver(tmp_path):
    out = run("fieldcool", "-o", tmp_path, "-s", 3, 2, "--J1", 1, "-B", 0, 0, 0.5, "--T_cold", 0.2, "--n_steps", 8,
              "--n_sweep", 4, "--n_burn_in", 4, "--n_sample", 3, "--init_uniform")
    assert "Releasing field" in out
    with File(only(tmp_path, ".out.h5")) as f:
        assert len(f["/energy/T_list"]) == 8
        assert list(f["/ssf/n_samples"]) == [3]
        assert f["/ssf/static_corr"].shape == (3, 1, 8, 2)


def test_resolved_ssf_from_the_drivers(tmp_path):
    """anneal and temper with --ssf_resolved: /ssf/static_corr in the
    sublattice-resolved layout [n_corr, n_T, n_k, 16, 16, 2] (src/temper.cpp:121-159),
    whose phase contraction is the contracted S(q) of the same run."""
    from oracle import ssf_fft
    base = ["-s", 5, 2, "--J1", 1, "--T_sample", 0.5, "--n_steps", 4, "--n_sweep", 2, "--n_burn_in", 2,
            "--n_sample", 2, "--init_uniform", "--correlators", "xx", "xy"]
    outs = {}
    for tag, extra in (("c", []), ("r", ["--ssf_resolved"])):
        d = tmp_path / tag
        d.mkdir()
        run("anneal", "-o", d, *base, *extra)
        with File(only(d, ".out.h5")) as f:
            outs[tag] = f["/ssf/static_corr"][:]
    c, r = outs["c"], outs["r"]
    assert c.shape == (2, 1, 8, 2) and r.shape == (2, 1, 8, 16, 16, 2)
    L = 2
    K = np.stack(np.meshgrid(np.arange(L), np.arange(L), np.arange(L), indexing="ij"), -1).reshape(-1, 3)
    dr = ssf_fft.R_SL[:, None, :] - ssf_fft.R_SL[None, :, :]
    ph = np.exp(1j * 2 * np.pi * np.einsum("kd,mnd->kmn", K, dr) / (8 * L))
    Sq = np.einsum("ctkmn,kmn->ctk", r[..., 0] + 1j * r[..., 1], ph)
    np.testing.assert_allclose(Sq.real, c[..., 0], atol=1e-6 * np.abs(c).max())
    np.testing.assert_allclose(Sq.imag, c[..., 1], atol=1e-6 * np.abs(c).max())
    d = tmp_path / "t"
    d.mkdir()
    run("temper", "-o", d, "-s", 3, "--n_replicas", 4, 2, "--J1", 1, "--T_sample", 0.3, "--n_sweep", 2,
        "--n_burn_in", 2, "--n_sample", 3, "--init_uniform", "--ssf_resolved")
    with File(only(d, ".out.h5")) as f:
        assert f["/ssf/static_corr"].shape == (3, 1, 8, 16, 16, 2)
        assert (f["/ssf/static_corr_2"][..., 0] >= 0).all()


def test_ltgs_driver(tmp_path):
    """ltgs (src/luttinger_tisza.cpp) with the k sweep on the GPU: printed lines,
    output tree, and E_min / k* against the oracle's numpy restatement."""
    import oracle.lt as olt
    out = run("ltgs", "-o", tmp_path, 3, "--J1", 1, "--J2", 0.1, "--J3", -0.05, "--Delta", 0.5)
    assert "LT minimum:" in out and "k*  idx" in out and "Saved to" in out
    e_ref, k_ref = olt.lt_minimum(3, 1.0, 0.1, -0.05, 0.5)
    with File(only(tmp_path, "ltgs.out.h5")) as f:
        assert abs(float(f["/E_min"]) - e_ref) <= 1e-9
        lam = f["/eigenvalue_map"][:]
        assert lam.shape == (27,) and abs(lam.min() - 2 * e_ref) <= 1e-9
        assert tuple(f["/k_star_idx"][:]) == tuple(k_ref)
        assert f["/eigenvector"].shape == (48, 2)
        np.testing.assert_allclose(f["/k_star_vec"][:], 2 * np.pi * np.array(k_ref) / 24.0)
        assert (f["/geometry/index_cell"] == 24 * np.eye(3)).all()
        assert list(f.attrs["k_dims"]) == [3, 3, 3]


@pytest.mark.parametrize("n_sweep,ssf_every", [(32, 16), (20, 16), (5, 0), (0, 16)])
def test_step_host_matches_the_same_calls(n_sweep, ssf_every):
    """pc_step_host (host spins in and out, the result copy overlapped with the
    last S(q) sample and the energy on a second stream) against the same work
    through separate calls: spins, energy, accepted moves and S(q) sums
    identical, twice in a row (the second call reuses its staging)."""
    L, T = 8, 0.7
    kw = dict(J1=1.0, J2=0.1, J3=0.05, B=(0.0, 0.0, 0.5), seed=31, schedule=1)
    a = pc.pyrochlore_system(L, **kw)
    b = pc.pyrochlore_system(L, **kw)
    for s in (a, b):
        s.ssf_configure(["xx", "zz", "xy"], 1)
    a.random_spins(2)
    S_in = np.ascontiguousarray(a.spins_f4())
    for _ in range(2):
        S_out = np.zeros_like(S_in)
        e, acc = a.step_host(S_in, S_out, T, n_sweep, ssf_every, 0 if ssf_every else -1)
        b.set_spins_f4(S_in)
        acc_b, done = 0, 0
        while done < n_sweep:
            k = min(ssf_every, n_sweep - done) if ssf_every else n_sweep
            acc_b += int(b.sweep([T], k, 1)[0])
            done += k
            if ssf_every and k == ssf_every:
                b.ssf_sample([0])
        e_b, _ = b.energy()
        np.testing.assert_array_equal(S_out, b.spins_f4())
        assert e == e_b[0]
        assert acc == acc_b
        for x, y in zip(a.ssf_read(0), b.ssf_read(0)):
            np.testing.assert_array_equal(np.asarray(x), np.asarray(y))
        S_in = S_out


@pytest.mark.parametrize("L", [2, 4, 8])
def test_spin_ft_matches_oracle_sublattice_dft(L):
    """pc_spin_ft (save_ft_spin_state's array, src/MC.cpp:320-368) against the
    numpy restatement of the per-sublattice DFT (itself pinned on the
    oracle's correlate); 1e-5 relative to the largest amplitude."""
    from oracle import ssf_fft
    g = pc.pyrochlore_system(L, J1=1.0, seed=1)
    g.random_spins(L)
    ft = g.spin_ft()
    ref = ssf_fft.sublattice_ft(g.spins(), L)
    assert ft.shape == (3, 16, L ** 3, 2)
    scale = np.abs(ref).max()
    assert np.abs(ft[..., 0] - ref.real).max() <= 1e-5 * scale
    assert np.abs(ft[..., 1] - ref.imag).max() <= 1e-5 * scale


def test_anneal_save_state_ft(tmp_path):
    args = ["-o", tmp_path, "-s", 5, 4, "--J1", 1, "--T_sample", 0.5, "--n_steps", 4, "--n_sweep", 2,
            "--n_burn_in", 2, "--n_sample", 2, "--init_uniform", "--save_state", "--save_state_ft"]
    out = run("anneal", *args)
    assert "Saving spin state FT" in out
    from oracle import ssf_fft
    with File(only(tmp_path, ".spins.h5")) as f:
        S = f["/spin_orientation"][:]
    with File(only(tmp_path, ".spindft.h5")) as f:
        ft = f["/spin_ft"][:]
    assert ft.shape == (3, 16, 64, 2)
    ref = ssf_fft.sublattice_ft(S, 4)
    assert np.abs(ft[..., 0] + 1j * ft[..., 1] - ref).max() <= 1e-5 * np.abs(ref).max()


def test_anneal_npz_container_holds_the_same_tree(tmp_path):
    """--npz writes the tree of the HDF5 output as an .npz archive: same
    datasets, shapes, values and attributes for the same seed."""
    args = ["-s", 11, 2, "--J1", 1, "--J2", 0.05, "--T_sample", 1.0, 0.5, "--n_steps", 6, "--n_sweep", 2,
            "--n_burn_in", 2, "--n_sample", 2, "--init_uniform", "--save_state"]
    (tmp_path / "h").mkdir()
    (tmp_path / "z").mkdir()
    run("anneal", "-o", tmp_path / "h", *args)
    run("anneal", "-o", tmp_path / "z", *args, "--npz")
    with File(only(tmp_path / "h", ".out.h5")) as a, File(only(tmp_path / "z", ".out.npz")) as b:
        for g in ("energy", "ssf", "geometry"):
            assert set(a[g].keys()) == set(b[g].keys()), g
            for k in a[g].keys():
                x, y = a[g + "/" + k][:], b[g + "/" + k][:]
                if x.dtype == object:
                    assert [s.decode() for s in x] == [s.decode() for s in y]
                else:
                    assert x.dtype == y.dtype and x.shape == y.shape, (g, k)
                    np.testing.assert_array_equal(x, y)
        for k in ("n_spins", "k_dims"):
            np.testing.assert_array_equal(a["ssf"].attrs[k], b["ssf"].attrs[k])
    with File(only(tmp_path / "h", ".spins.h5")) as a, File(only(tmp_path / "z", ".spins.npz")) as b:
        np.testing.assert_array_equal(a["/spin_orientation"][:], b["/spin_orientation"][:])


def test_anneal_file_holds_finished_temperatures_while_running(tmp_path):
    """The reference pre-allocates /ssf/static_corr and writes each sample
    temperature's slice when its sampling ends (include/ssf_manager.hpp:375-465),
    so an interrupted run leaves a readable file with the temperatures finished
    so far. The driver is paused (SIGSTOP: its host thread stops, kernels
    already queued finish) when it starts sampling the second temperature; the
    file on disk then holds the first temperature's slice and zeros in the
    others, and no /ssf/T_list yet. After SIGCONT the run completes normally."""
    import signal

    build.build()
    exe = os.path.join(build.BIN, "anneal")
    args = ["-o", tmp_path, "-s", 3, 4, "--J1", 1, "--J2", -0.1, "--T_sample", 1.0, 0.5, 0.2, "--n_steps", 30,
            "--n_sweep", 4, "--n_burn_in", 4, "--n_sample", 4, "--init_uniform"]
    p = subprocess.Popen(["stdbuf", "-oL", exe, *map(str, args)], stdout=subprocess.PIPE, text=True)
    seen = 0
    stopped = False
    try:
        for line in p.stdout:
            if line.startswith("Sampling at T"):
                seen += 1
                if seen == 2:
                    os.kill(p.pid, signal.SIGSTOP)
                    stopped = True
                    break
        assert stopped
        with File(only(tmp_path, ".out.h5")) as f:
            sc = f["/ssf/static_corr"][:]
            assert "/ssf/T_list" not in f
        assert sc.shape == (6, 3, 64, 2)
        # T_sample sorted ascending: slot 2 is T = 1.0, sampled first
        assert np.abs(sc[:, 2]).max() > 0
        assert np.abs(sc[:, :2]).max() == 0
    finally:
        if stopped:
            os.kill(p.pid, signal.SIGCONT)
        p.stdout.read()
        p.wait(timeout=300)
    assert p.returncode == 0
    with File(only(tmp_path, ".out.h5")) as f:
        sc = f["/ssf/static_corr"][:]
        np.testing.assert_array_equal(f["/ssf/T_list"][:], [0.2, 0.5, 1.0])
    assert (np.abs(sc).reshape(6, 3, -1).max(axis=2) > 0).all()


@pytest.mark.parametrize("update", [0, 1])
def test_step_host3_matches_step_host(update):
    """pc_step_host3 (packed x, y, z host spins, unpacked and packed on the
    device) against pc_step_host on the same spins: the same spins out, energy,
    accepted moves and S(q) sums, over three consecutive steps. With lifted
    Metropolis (update 1) the lifting directions stay on the device: the float4
    path is fed its own output, directions included, and the chains agree."""
    L, T = 8, 0.7
    kw = dict(J1=1.0, J2=0.1, J3=0.05, B=(0.0, 0.0, 0.5), seed=37, schedule=1, update=update)
    a = pc.pyrochlore_system(L, **kw)
    b = pc.pyrochlore_system(L, **kw)
    for s in (a, b):
        s.ssf_configure(["xx", "zz", "xy"], 1)
    a.random_spins(4)
    S4 = np.ascontiguousarray(a.spins_f4())
    b.set_spins_f4(S4)
    S3 = np.ascontiguousarray(S4[:, :3])
    for _ in range(3):
        S3_out = np.zeros_like(S3)
        S4_out = np.zeros_like(S4)
        e3, acc3 = a.step_host3(S3, S3_out, T, 20, 8, 0)
        e4, acc4 = b.step_host(S4, S4_out, T, 20, 8, 0)
        np.testing.assert_array_equal(S3_out, S4_out[:, :3])
        assert e3 == e4 and acc3 == acc4
        S3, S4 = S3_out, S4_out
    for x, y in zip(a.ssf_read(0), b.ssf_read(0)):
        np.testing.assert_array_equal(np.asarray(x), np.asarray(y))
    np.testing.assert_array_equal(a.spins_f4(), b.spins_f4())
    with pytest.raises(ValueError):
        a.step_host3(np.zeros((a.N(0), 4), np.float32), S3, T, 1)
