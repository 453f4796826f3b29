"""Parity of the CUDA path (through the C ABI) with the FP64 oracle.

Tolerances (FP32 spins and transforms against an FP64 oracle):
  energy per cell, local fields, one overrelaxation pass, S(q): 1e-5 relative
  to the scale of the quantity (max |value| over the array);
  trajectories of a few sweeps: 1e-4 absolute per spin component;
  integer tables: exact.
"""
import numpy as np
import pytest

import oracle
import pyro_cmc_b200 as pc

pytestmark = pytest.mark.gpu

REL = 1e-5

COUPLINGS = [
    dict(J1=1.0, J2=0.0, J3=0.0, Delta=1.0, B=(0.0, 0.0, 0.0)),
    dict(J1=1.0, J2=-0.1, J3=0.05, Delta=1.0, B=(0.0, 0.0, 0.0)),
    dict(J1=1.0, J2=0.1, J3=-0.05, Delta=0.5, B=(0.2, 0.0, 0.0)),
    dict(J1=-0.7, J2=0.3, J3=0.02, Delta=1.3, B=(0.0, 0.1, 0.5)),
]


def pair(L, c, seed=0, colouring=0, **kw):
    g = pc.pyrochlore_system(L, seed=seed, colouring=colouring, **c, **kw)
    assert g.structured() != bool(kw.get("generic", False))
    o = oracle.System(L, seed=seed, **c)
    return g, o


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def states(o, rng):
    _, sl = o.positions()
    pos, _ = o.positions()
    z = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], float) / np.sqrt(3)
    q = 2 * np.pi * 3 / (8 * o.L)
    spiral = np.stack([np.zeros(len(pos)), np.cos(q * pos[:, 2]), np.sin(q * pos[:, 2])], axis=1)
    fm = np.tile([0.48, 0.6, 0.64], (o.N, 1))
    return {"random": unit(rng, o.N), "fm": fm, "aiao": z[sl % 4], "spiral": spiral}


@pytest.mark.parametrize("L", [1, 2, 3, 5])
def test_neighbour_tables_bit_exact(L):
    g, o = pair(L, COUPLINGS[1])
    assert o.num_specs() == len(g.spec_names) == 9
    for spec in range(9):
        a = g.neighbour_table(spec, max_nb=16)
        b = o.neighbours(spec, max_nb=16)
        a = a[:, : b.shape[1]]
        np.testing.assert_array_equal(np.sort(a, axis=1), np.sort(b, axis=1))


def test_positions_match_oracle():
    g, o = pair(3, COUPLINGS[0])
    pg, sg = g.positions()
    po, so = o.positions()
    np.testing.assert_array_equal(pg, po % 24)
    np.testing.assert_array_equal(sg, so)


@pytest.mark.parametrize("generic", [False, True])
@pytest.mark.parametrize("L", [1, 2, 4, 8])
@pytest.mark.parametrize("ci", range(len(COUPLINGS)))
def test_energy_and_local_field(L, ci, generic):
    g, o = pair(L, COUPLINGS[ci], generic=generic)
    rng = np.random.default_rng(100 * L + ci)
    for name, S in states(o, rng).items():
        o.set_spins(S)
        g.set_spins(S)
        S32 = g.spins()  # what the device holds (FP32)
        o.set_spins(S32)
        e_ref = o.energy()
        h_ref = o.local_fields()
        e, m = g.energy()
        scale = 16 * (6 * abs(COUPLINGS[ci]["J1"]) + 12 * abs(COUPLINGS[ci]["J2"]) + 12 * abs(COUPLINGS[ci]["J3"]) + 1)
        assert abs(e[0] - e_ref) <= REL * scale, (name, e[0], e_ref)
        np.testing.assert_allclose(m[0], S32.sum(axis=0), atol=1e-6 * o.N)
        h = g.local_field()
        err = np.abs(h - h_ref).max() / max(1.0, np.abs(h_ref).max())
        assert err <= REL, (name, err)


@pytest.mark.parametrize("L", [1, 2, 4])
@pytest.mark.parametrize("J2", [-0.1, 0.0])
@pytest.mark.parametrize("uniform", [True, False])
def test_isotropic_energy_per_group_and_per_bond_sums(L, J2, uniform):
    """Isotropic couplings: with each group's j the same on every sublattice
    the per-cell energy sums bare S_i.S_j per group and applies j once per
    cell; with one J1 pair's j changed (1.3 on pyrochlore sublattices 0-1) it
    applies each bond's j. Both (and J2 = 0, whose group is skipped) against
    the FP64 sum over the oracle's neighbour tables with the same matrices."""
    c = dict(J1=1.0, J2=J2, J3=0.05, Delta=1.0, B=(0.1, 0.0, 0.3))
    g, o = pair(L, c)
    mats = [o.spec_matrix(k) for k in range(o.num_specs())]
    if not uniform:
        mats[0] = 1.3 * np.eye(3)
        g.set_coupling_matrix(0, mats[0])
    assert g.structured()
    rng = np.random.default_rng(7 * L + (J2 != 0) + 2 * uniform)
    for name, S in states(o, rng).items():
        g.set_spins(S)
        S32 = g.spins().astype(np.float64)
        h = np.zeros_like(S32)
        for k, M in enumerate(mats):
            nb = o.neighbours(k)
            for col in range(nb.shape[1]):
                idx = nb[:, col]
                ok = idx >= 0
                h[ok] += S32[idx[ok]] @ M.T
        e_ref = (0.5 * np.sum(S32 * h) - np.sum(S32 @ np.array(c["B"]))) / L**3
        e, m = g.energy()
        scale = 16 * (6 * 1.3 + 12 * abs(J2) + 12 * 0.05 + 1)
        assert abs(e[0] - e_ref) <= REL * scale, (name, e[0], e_ref)
        np.testing.assert_allclose(m[0], S32.sum(axis=0), atol=1e-6 * o.N)


def test_ferromagnet_energy_known_answer():
    c = dict(J1=1.3, J2=-0.4, J3=0.25, Delta=1.0, B=(0.1, -0.2, 0.7))
    g = pc.pyrochlore_system(4, **c)
    n = np.array([0.48, 0.6, 0.64])
    g.set_spins(np.tile(n, (g.N(), 1)))
    e, _ = g.energy()
    exact = 48 * 1.3 + 96 * -0.4 + 96 * 0.25 - 16 * np.dot([0.1, -0.2, 0.7], n)
    assert e[0] == pytest.approx(exact, rel=1e-5)


@pytest.mark.parametrize("colouring", [0, 1])
@pytest.mark.parametrize("ci", [0, 2])
def test_overrelax_pass_with_given_angles(colouring, ci):
    g, o = pair(4, COUPLINGS[ci], colouring=colouring)
    rng = np.random.default_rng(7)
    S = unit(rng, o.N)
    g.set_spins(S)
    o.set_spins(g.spins())
    _, col = g.colours()
    theta = rng.uniform(0, 2 * np.pi, o.N)
    e0 = o.energy()
    g.overrelax_theta(theta)
    o.overrelax(theta, colour_of_sl=col)
    _close_fp32(g.spins(), o.spins())
    e, _ = g.energy()
    assert e[0] == pytest.approx(e0, abs=1e-4)
    g.overrelax_theta(None)  # reflection
    o.overrelax(None, colour_of_sl=col)
    _close_fp32(g.spins(), o.spins())


def _close_fp32(a, b):
    """One FP32 overrelaxation pass against FP64: the rotation axis is the
    local field, a sum of up to 30 unit vectors in FP32 (error ~1e-6 of the
    sum's scale); where those nearly cancel (|h| << 1) the axis direction, and
    with it the rotated spin, carries a larger relative error. Bound: 99.5% of
    components within 1e-5, all within 2e-4."""
    d = np.abs(a - b)
    assert np.mean(d <= 1e-5) >= 0.995, np.sort(d.ravel())[-10:]
    assert d.max() <= 2e-4


def test_colour_classes():
    g = pc.pyrochlore_system(2, J1=1.0, J2=0.1, J3=0.0, colouring=1)
    n, col = g.colours()
    assert n == 4 and (col == np.arange(16) % 4).all()
    g = pc.pyrochlore_system(2, J1=1.0, J2=0.1, J3=0.05, colouring=1)
    n, col = g.colours()
    assert n == 16
    g = pc.pyrochlore_system(2, J1=1.0, colouring=0)
    n, col = g.colours()
    assert n == 16 and (col == np.arange(16)).all()


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("path", ["generic", "v0", "v1", "v2", "v3"])
@pytest.mark.parametrize("colouring", [0, 1])
@pytest.mark.parametrize("T", [0.3, 2.0])
def test_sweeps_follow_oracle_mirror(colouring, T, path, schedule):
    c = COUPLINGS[2]
    seed = 12345
    g, o = pair(3, c, seed=seed, colouring=colouring, generic=(path == "generic"), schedule=schedule)
    if path != "generic":
        g.set_load_variant(int(path[1]))
    rng = np.random.default_rng(3)
    g.set_spins(unit(rng, o.N))
    o.set_spins(g.spins())
    _, col = g.colours()
    for sweep in range(3):
        acc_g = g.sweep(T, 1, 1)[0]
        acc_o = o.sweep_philox(T, seed, 0, sweep, col, n_overrelax=1, or_mode=0, fused=bool(schedule))
        Sg = g.spins()
        So = o.spins()
        assert int(acc_g) == int(acc_o)
        np.testing.assert_allclose(Sg, So, atol=1e-4)
        o.set_spins(Sg)  # re-sync to FP32 state
    assert g.sweep_counter() == 3


@pytest.mark.parametrize("schedule", [0, 1])
def test_sweep_reflection_mode_follows_oracle(schedule):
    c = COUPLINGS[1]
    seed = 99
    g, o = pair(2, c, seed=seed, overrelax_mode=1, schedule=schedule)
    rng = np.random.default_rng(5)
    g.set_spins(unit(rng, o.N))
    o.set_spins(g.spins())
    _, col = g.colours()
    acc_g = g.sweep(0.7, 1, 2)[0]
    acc_o = o.sweep_philox(0.7, seed, 0, 0, col, n_overrelax=2, or_mode=1, fused=bool(schedule))
    assert int(acc_g) == int(acc_o)
    # two reflections about FP32 local fields: each roughly doubles the axis
    # error of sites whose field nearly cancels
    d = np.abs(g.spins() - o.spins())
    assert np.mean(d <= 1e-4) >= 0.95 and d.max() <= 1e-3


def _close_rounding(a, b):
    """Two FP32 chains that differ only in rounding, a few sweeps apart:
    99.5 % of the components within 1e-5, all within 1e-3 (an overrelaxation
    about a nearly cancelling field amplifies a last-bit difference)."""
    d = np.abs(np.asarray(a, float) - np.asarray(b, float))
    assert (d <= 1e-5).mean() >= 0.995, (d <= 1e-5).mean()
    assert d.max() <= 1e-3, d.max()


def _sweep_state(L, n, setup, c=COUPLINGS[1], schedule=1):
    g = pc.pyrochlore_system(L, seed=4, schedule=schedule, **c)
    g.random_spins(9)
    setup(g)
    acc = g.sweep(0.7, n, 1)
    return g.spins_f4(), acc


@pytest.mark.parametrize("schedule", [0, 1])
def test_launch_modes_give_identical_sweeps(schedule):
    """Graphs of up to 16 sweeps (37 = 16 + 16 + 5), plain launches with
    per-kernel events, launch overlap on and off, a strided grid and one CTA
    per tile: the same moves, bit for bit."""
    L, n = 6, 37
    ref, acc_ref = _sweep_state(L, n, lambda g: g.set_kernel_timing(True), schedule=schedule)
    for setup in (lambda g: None,
                  lambda g: g.set_launch_overlap(False),
                  lambda g: g.set_tile(64, 0),
                  lambda g: g.set_tile(128, 3)):
        S, acc = _sweep_state(L, n, setup, schedule=schedule)
        assert np.array_equal(S, ref)
        assert np.array_equal(acc, acc_ref)


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("threads", [64, 256])
def test_staged_rows_match_per_site_kernel(schedule, threads):
    """Load variant 3 (neighbour rows staged by bulk copies) against the
    per-site kernel over two sweeps: the same moves up to FP32 rounding (the
    two kernels may contract the arithmetic differently, and a chaotic chain
    amplifies a last-bit difference over many sweeps)."""
    L, n = 6, 2
    ref, acc_ref = _sweep_state(L, n, lambda g: g.set_tile(threads, 0), schedule=schedule)
    S, acc = _sweep_state(L, n, lambda g: (g.set_tile(threads, 0), g.set_load_variant(3)), schedule=schedule)
    _close_rounding(S, ref)
    assert np.array_equal(acc, acc_ref)


def test_mixed_sizes_staged_rows():
    """Replicas of different L in one launch (row tiles of different shapes,
    a ragged last tile for L = 12): the staged kernel makes the same moves as
    the per-site kernel, up to FP32 rounding."""
    Ls = [3, 8, 5, 12]
    out = []
    for variant in (0, 3):
        g = pc.pyrochlore_system(Ls, seed=6, schedule=1, **COUPLINGS[1])
        g.set_load_variant(variant)
        g.random_spins(4)
        acc = g.sweep(0.9, 2, 1)
        out.append((acc, [g.spins_f4(r) for r in range(len(Ls))]))
    assert np.array_equal(out[0][0], out[1][0])
    for a, b in zip(out[0][1], out[1][1]):
        _close_rounding(a, b)


def test_batched_replicas_are_independent_streams():
    c = COUPLINGS[1]
    g = pc.pyrochlore_system(2, seed=5, n_replicas=3, **c)
    rng = np.random.default_rng(1)
    S = unit(rng, g.N())
    for r in range(3):
        g.set_spins(S, r)
    g.sweep([0.5, 0.5, 0.5], 2, 1)
    o = oracle.System(2, seed=5, **c)
    for r in range(3):
        o.set_spins(S.astype(np.float32).astype(np.float64))
        o.sweep_philox(0.5, 5, r, 0, np.arange(16), 1)
        o.sweep_philox(0.5, 5, r, 1, np.arange(16), 1)
        np.testing.assert_allclose(g.spins(r), o.spins(), atol=2e-4)
    assert np.abs(g.spins(0) - g.spins(1)).max() > 0.1


def test_spins_stay_normalised_over_many_sweeps():
    g = pc.pyrochlore_system(4, J1=1.0, J2=0.1, J3=0.05, B=(0, 0, 0.3))
    g.random_spins(3)
    g.sweep(0.1, 200, 1)
    S = g.spins()
    assert np.abs(np.linalg.norm(S, axis=1) - 1).max() < 1e-5


def test_random_spins_uniform_on_sphere():
    g = pc.pyrochlore_system(8, J1=1.0)
    g.random_spins(42)
    S = g.spins()
    assert np.abs(np.linalg.norm(S, axis=1) - 1).max() < 1e-5
    assert np.abs(S.mean(axis=0)).max() < 0.02
    assert np.abs((S ** 2).mean(axis=0) - 1 / 3).max() < 0.02


CORR9 = ["xx", "yy", "zz", "xy", "xz", "yz", "yx", "zx", "zy"]


@pytest.mark.parametrize("L", [1, 2, 3, 4, 6, 8, 12])
def test_ssf_matches_oracle(L):
    g, o = pair(L, COUPLINGS[0])
    g.ssf_configure(CORR9, 1)
    rng = np.random.default_rng(L)
    for name, S in states(o, rng).items():
        g.set_spins(S)
        o.set_spins(g.spins())
        ref = o.ssf(CORR9, mode=0)
        got = g.ssf_current()
        # relative to the largest |S(q)|, and never below N (the size of S(q)
        # of an uncorrelated state): states such as all-in-all-out have
        # S(q) = 0 on the whole grid, where only an absolute bound means anything
        scale = max(np.abs(ref).max(), o.N)
        assert np.abs(got - ref).max() <= REL * scale, (name, np.abs(got - ref).max() / scale)


@pytest.mark.parametrize("L", [11, 12, 16, 24, 32, 64])
def test_ssf_large_L_matches_fft_restatement(L):
    """S(q) of random spins at sizes beyond the direct-sum oracle: L = 11
    (a prime line length, the runtime-radix path), 12 and 24 (the tempering
    ladder sizes, unswizzled), 16 / 32 / 64 (the swizzled shared-memory
    layout; 64 is the field-cool size), against the numpy-FFT restatement of
    ssf_manager::sample."""
    from oracle import ssf_fft
    g = pc.pyrochlore_system(L, **COUPLINGS[0])
    g.ssf_configure(CORR9, 1)
    g.random_spins(L)
    got = g.ssf_current()
    ref = ssf_fft.ssf(g.spins(), L, CORR9)
    scale = max(np.abs(ref).max(), g.N())
    assert np.abs(got - ref).max() <= REL * scale, np.abs(got - ref).max() / scale
    # structured state: a spiral along z concentrates S^yy + S^zz at one K
    pos, _ = g.positions()
    q = 2 * np.pi * 3 / (8 * L)
    spiral = np.stack([np.zeros(len(pos)), np.cos(q * pos[:, 2]), np.sin(q * pos[:, 2])], axis=1)
    g.set_spins(spiral)
    got = g.ssf_current()
    ref = ssf_fft.ssf(g.spins(), L, CORR9)
    scale = max(np.abs(ref).max(), g.N())
    assert np.abs(got - ref).max() <= REL * scale, np.abs(got - ref).max() / scale


def test_ssf_accumulates_like_ssf_manager():
    g, o = pair(4, COUPLINGS[0])
    g.ssf_configure(["xx", "yy", "zz", "xy"], 2)
    rng = np.random.default_rng(0)
    refs = []
    for k in range(3):
        S = unit(rng, o.N)
        g.set_spins(S)
        o.set_spins(g.spins())
        refs.append(o.ssf(["xx", "yy", "zz", "xy"]))
        g.ssf_sample([1])
    s, q, n = g.ssf_read(1)
    assert n == 3
    ref_s = sum(refs)
    ref_q = sum(r ** 2 for r in refs)
    assert np.abs(s - ref_s).max() <= REL * np.abs(ref_s).max()
    assert np.abs(q - ref_q).max() <= 3 * REL * np.abs(ref_q).max()
    s0, _, n0 = g.ssf_read(0)
    assert n0 == 0 and not s0.any()
    g.ssf_clear(1)
    s, _, n = g.ssf_read(1)
    assert n == 0 and not s.any()


def test_ssf_spiral_byhand_peaks():
    # spiral_byhand (test/spiral_byhand.cpp:100-107): S = (0, cos q.r, sin q.r)
    L = 4
    g = pc.pyrochlore_system(L, J1=-1.0, split_J1=False)
    g.ssf_configure(["xx", "yy", "zz"], 1)
    pos, _ = g.positions()
    Q = np.array([1, 2, 0])
    qv = 2 * np.pi * Q / (8 * L)
    ph = pos @ qv
    S = np.stack([np.zeros(len(ph)), np.cos(ph), np.sin(ph)], axis=1)
    g.set_spins(S)
    out = g.ssf_current()
    tot = out[1, :, 0] + out[2, :, 0]
    k_of = lambda K: ((K[0] % L) * L + (K[1] % L)) * L + (K[2] % L)
    N = g.N()
    # the helix puts N^2/2 at q = +Q; q = -Q is not on the K in [0,L)^3 grid
    # (K = -Q mod L differs from -Q by a vector that is not a reciprocal
    # vector of the site positions, so the sublattice phases do not repeat)
    assert tot[k_of(Q)] == pytest.approx(N * N / 2, rel=1e-5)
    assert np.abs(out[0]).max() < 1e-3 * N
    mask = np.ones_like(tot, bool)
    mask[k_of(Q)] = False
    assert np.abs(tot[mask]).max() < 1e-3 * N * N
    # energy against the oracle with the same single-J1 spec
    o = oracle.System(L, J1=-1.0, j1_mode=1)
    o.set_spins(g.spins())
    e, _ = g.energy()
    assert e[0] == pytest.approx(o.energy(), abs=1e-5 * 96)


def test_invalid_correlator_names_raise():
    g = pc.pyrochlore_system(2, J1=1.0)
    with pytest.raises(pc.InvalidArgument, match="unknown spin component"):
        g.ssf_configure(["xq"], 1)
    with pytest.raises(pc.InvalidArgument, match="2 chars"):
        g.ssf_configure(["xyz"], 1)


def test_duplicate_coupling_name_raises():
    g = pc.System(2)
    g.define_pyrochlore(1.0)
    with pytest.raises(pc.InvalidArgument, match="unique"):
        g.define_coupling("J2", [[], [], [], []], np.eye(3))


def test_coupling_matrices_set_at_once_match_one_by_one():
    """pc_set_coupling_matrices (one rebuild of the tables) gives the energy
    and local fields of the same matrices set one at a time, against the FP64
    sum over the oracle's neighbour tables; setting the values it already
    holds changes nothing, and an index out of range changes nothing either."""
    c = COUPLINGS[1]
    a, o = pair(4, c)
    b = pc.pyrochlore_system(4, **c)
    specs = [0, 3, 6, 8]
    mats = [1.3 * np.eye(3), 0.7 * np.eye(3), 0.2 * np.eye(3), -0.1 * np.eye(3)]
    for k, M in zip(specs, mats):
        a.set_coupling_matrix(k, M)
    b.set_coupling_matrices(specs, mats)
    b.set_coupling_matrices(specs, mats)
    S = unit(np.random.default_rng(5), o.N)
    for s in (a, b):
        s.set_spins(S)
    assert a.structured() and b.structured()
    np.testing.assert_array_equal(a.energy()[0], b.energy()[0])
    np.testing.assert_array_equal(a.local_field(), b.local_field())
    full = [o.spec_matrix(k) for k in range(o.num_specs())]
    for k, M in zip(specs, mats):
        full[k] = M
    S32 = b.spins().astype(np.float64)
    h = np.zeros_like(S32)
    for k, M in enumerate(full):
        nb = o.neighbours(k)
        for col in range(nb.shape[1]):
            idx = nb[:, col]
            ok = idx >= 0
            h[ok] += S32[idx[ok]] @ M.T
    e_ref = 0.5 * np.sum(S32 * h) / 4**3
    assert abs(b.energy()[0][0] - e_ref) <= REL * 16 * (6 * 1.3 + 12 + 1)
    with pytest.raises(pc.InvalidArgument):
        b.set_coupling_matrices([0, 99], [np.eye(3), np.eye(3)])
    np.testing.assert_array_equal(a.energy()[0], b.energy()[0])


def test_nonstructural_coupling_uses_generic_path():
    # an asymmetric J2 gives the J2 group two different matrices (J on the
    # source side, J^T on the target side): the generic tables must take over
    g = pc.System(2)
    g.define_pyrochlore(1.0, 0.0, 0.0)
    g.setup_lattice()
    assert g.structured()
    g.set_coupling_matrix(6, [[0.1, 0.05, 0.0], [0.0, 0.1, 0.0], [0.0, 0.0, 0.1]])
    assert not g.structured()


@pytest.mark.parametrize("L", [1, 2, 3, 4])
def test_ssf_resolved_matches_oracle_correlate(L):
    """The sublattice-resolved correlator (ssf_manager's correlate() output)
    against the oracle's per-sublattice DFT, 9 correlators, random spins."""
    g, o = pair(L, COUPLINGS[0])
    g.ssf_set_resolved(True)
    g.ssf_configure(CORR9, 1)
    rng = np.random.default_rng(L + 40)
    g.set_spins(unit(rng, o.N))
    o.set_spins(g.spins())
    got = g.ssf_current()
    _, ref = o.ssf(CORR9, mode=1, resolved=True)
    scale = max(np.abs(ref).max(), 1.0)
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= REL * scale * 10, np.abs(got - ref).max() / scale


@pytest.mark.parametrize("L", [6, 8, 16])
def test_ssf_resolved_contracts_to_ssf(L):
    """Contracting the resolved correlator with exp(+i q.(r_mu - r_nu)) gives
    S(q) (include/ssf_manager.hpp:275-280); accumulation in slots as
    ssf_manager does (two samples)."""
    from oracle import ssf_fft
    corr = ["xx", "zz", "xy", "yz"]
    g = pc.pyrochlore_system(L, **COUPLINGS[0])
    g.ssf_set_resolved(True)
    g.ssf_configure(corr, 2)
    refs = []
    for k in range(2):
        g.random_spins(100 + k)
        refs.append(ssf_fft.ssf(g.spins(), L, corr))
        g.ssf_sample([1])
    s, q, n = g.ssf_read(1)
    assert n == 2 and s.shape == (len(corr), L ** 3, 16, 16, 2)
    K = np.stack(np.meshgrid(np.arange(L), np.arange(L), np.arange(L), indexing="ij"), -1).reshape(-1, 3)
    dr = ssf_fft.R_SL[:, None, :] - ssf_fft.R_SL[None, :, :]  # [mu][nu][3]
    ph = np.exp(1j * 2 * np.pi * np.einsum("kd,mnd->kmn", K, dr) / (8 * L))
    C = s[..., 0] + 1j * s[..., 1]
    Sq = np.einsum("ckmn,kmn->ck", C, ph)
    ref = refs[0] + refs[1]
    scale = np.abs(ref).max()
    assert np.abs(Sq.real - ref[..., 0]).max() <= 1e-5 * scale
    assert np.abs(Sq.imag - ref[..., 1]).max() <= 1e-5 * scale
    assert (q[..., 0] >= 0).all() and (q[..., 1] >= 0).all()
    with pytest.raises(pc.PyroCMCError):
        g.ssf_forward_device(0)  # the differentiable S(q) is the contracted one
