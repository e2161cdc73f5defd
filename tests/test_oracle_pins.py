"""The oracle against the reference's own known answers (CPU only).

The reference ships no golden data files; its tests pin the path through
analytic and exact properties.  Each test below restates one of them against
the oracle, citing the reference test it follows, which is what pins the
oracle before it is trusted as the GPU's checker.
"""
import math

import numpy as np
import pytest

from legendre_b200 import rng as host_rng
from util import centers, relative_eq, with_ghosts

H = 0.4


# ------------------------------------------------------------------ rng ----
def test_splitmix64_known_answers(orc):
    # The published SplitMix64 generator seeded with 0 yields
    # 0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F first: the
    # reference's finalizer applied to k * 0x9E3779B97F4A7C15 must reproduce
    # that sequence.
    gamma = 0x9E3779B97F4A7C15
    expect = [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]
    for k, e in enumerate(expect):
        z = (k * gamma) & ((1 << 64) - 1)
        assert orc.splitmix64(z) == e
        assert host_rng.splitmix64(z) == e


def test_rng_deterministic_and_key_sensitive(orc):
    # src/util/rng.rs:55-63
    k = orc.mix_key(42, [7, 3, 1, 999])
    a = orc.standard_normal([k, k, k ^ 1])
    assert a[0] == a[1]
    assert a[0] != a[2]
    assert host_rng.mix_key(42, [7, 3, 1, 999]) == k


def test_rng_moments_are_standard_normal(orc):
    # src/util/rng.rs:65-78: 2e5 deviates keyed mix_key(1234, [i])
    keys = np.array([orc.mix_key(1234, [i]) for i in range(200_000)], dtype=np.uint64)
    x = orc.standard_normal(keys)
    mean = x.sum() / x.size
    var = (x * x).sum() / x.size - mean * mean
    assert abs(mean) < 0.01
    assert abs(var - 1.0) < 0.02


def test_unit_open_is_never_zero():
    assert host_rng.unit_open(0) == 1.0 / 9007199254740992.0
    assert host_rng.unit_open((1 << 64) - 1) == 1.0


# ----------------------------------------------------------------- ghosts --
def _global_index_state(orc, cells, block, ghost, periodic=None):
    g = orc.Grid(cells, block, [0.0] * len(cells), [1.0] * len(cells), periodic)
    st = orc.State(g, [ghost])
    x = centers(cells, block, [0.0] * len(cells), [1.0] * len(cells), 0) - 0.5
    if len(cells) == 2:
        y = centers(cells, block, [0.0, 0.0], [1.0, 1.0], 1) - 0.5
        x = 10.0 * y + x  # u(i, j) = 10 j + i (exact)
    st.set(0, with_ghosts(x, ghost))
    st.fill_ghosts(0)
    return st.get(0)


def test_halo_and_mirror_values_are_exact(orc):
    # tests/framework.rs:91-114
    v = _global_index_state(orc, [8], [4], 1)
    assert v[0][0] == 0.0 and v[1][5] == 7.0   # mirror
    assert v[0][5] == 4.0 and v[1][0] == 3.0   # exchange


def test_wide_ghosts_fill_every_layer(orc):
    # tests/framework.rs:117-138 (ghost width 2: index k sits at k + 2)
    v = _global_index_state(orc, [8], [4], 2)
    assert v[0][1] == 0.0 and v[0][0] == 1.0
    assert v[0][6] == 4.0 and v[0][7] == 5.0


def test_periodic_ghosts_across_blocks(orc):
    # tests/periodic.rs:72-92
    v = _global_index_state(orc, [8], [4], 1, [True])
    assert v[0][5] == 4.0 and v[1][0] == 3.0
    assert v[0][0] == 7.0 and v[1][5] == 0.0


def test_single_block_self_wrap(orc):
    # tests/periodic.rs:96-112
    v = _global_index_state(orc, [4], [4], 2, [True])
    assert v[0][1] == 3.0 and v[0][0] == 2.0 and v[0][6] == 0.0 and v[0][7] == 1.0


def test_mixed_periodic_and_mirror_corners(orc):
    # tests/periodic.rs:116-142; slabs are [block][j+1][i+1]
    v = _global_index_state(orc, [4, 4], [4, 4], 1, [True, False])[0]
    at = lambda i, j: v[j + 1][i + 1]
    assert at(-1, 0) == 3.0 and at(4, 2) == 20.0
    assert at(1, -1) == 1.0 and at(2, 4) == 32.0
    assert at(-1, -1) == 3.0 and at(4, 4) == 30.0


def test_face_neighbor_wraps_only_periodic_dimensions(orc):
    # tests/periodic.rs:41-66
    g = orc.Grid([4, 4], [2, 2], [0.0, 0.0], [1.0, 1.0], [True, False])
    assert g.face_neighbor(0, 0, 1) == 1
    assert g.face_neighbor(0, 0, -1) == 1 and g.face_neighbor(1, 0, 1) == 0
    assert g.face_neighbor(0, 1, -1) is None and g.face_neighbor(2, 1, 1) is None
    one = orc.Grid([4], [4], [0.0], [1.0], [True])
    assert one.face_neighbor(0, 0, 1) == 0 and one.face_neighbor(0, 0, -1) == 0


def test_cell_centers(orc):
    # tests/framework.rs:60-66
    g = orc.Grid([4], [2], [10.0], [0.5])
    assert g.cell_center(0, [0]) == (10.25,)
    assert g.cell_center(1, [1]) == (11.75,)


# ------------------------------------------------------------------- heat --
def _heat_mode(orc, cells, block, h, kappa, dt, steps, periodic=None, full_period=False):
    D = len(cells)
    g = orc.Grid(cells, block, [0.0] * D, [h] * D, periodic)
    st = orc.State(g, [1])
    n = cells[0]
    kx = (2.0 if full_period else 1.0) * math.pi / (n * h)
    x = centers(cells, block, [0.0] * D, [h] * D, 0)
    u0 = np.vectorize(math.cos)(kx * x)
    st.set(0, with_ghosts(u0, 1))
    st.heat_run(0, kappa, 0.0, dt, steps)
    lam = math.fma(2.0, -math.cos(kx * h), 2.0) if hasattr(math, "fma") else 2.0 - 2.0 * math.cos(kx * h)
    lam = lam / (h * h)
    factor = (1.0 - dt * kappa * lam) ** steps
    return st.interior(0), factor * u0


def test_heat3d_matches_discrete_eigenmode_decay(orc):
    # tests/heat3d.rs:82-137: 16^3 as 2x2x2 blocks, mirror, 200 steps
    h, kappa = 0.1, 0.7
    dt = 0.5 / 6.0 * h * h / kappa
    got, expected = _heat_mode(orc, [16] * 3, [8] * 3, h, kappa, dt, 200)
    assert relative_eq(got, expected, 1e-10, 1e-12).all()


def test_heat2d_matches_discrete_eigenmode_decay(orc):
    # tests/heat.rs:86-161: 32^2 as 4x4 blocks, dt = 0.25 h^2 / kappa
    h, kappa = 0.1, 0.7
    dt = 0.25 * (h * h) / kappa
    got, expected = _heat_mode(orc, [32, 32], [8, 8], h, kappa, dt, 200)
    assert relative_eq(got, expected, 1e-10, 1e-12).all()


@pytest.mark.parametrize("blocks_per_side", [1, 2])
def test_periodic_eigenmode_decays_exactly(orc, blocks_per_side):
    # tests/periodic.rs:223-284
    h, kappa = 0.1, 0.7
    dt = 0.25 * (h * h) / kappa
    got, expected = _heat_mode(orc, [32, 32], [32 // blocks_per_side] * 2, h, kappa, dt, 200, [True, True],
                               full_period=True)
    assert relative_eq(got, expected, 1e-10, 1e-12).all()


def test_heat_threads_bitwise_identical(orc):
    # tests/heat3d.rs:139-144 (RayonScheduler == SerialScheduler)
    h, kappa = 0.1, 0.7
    dt = 0.5 / 6.0 * h * h / kappa
    g = orc.Grid([16] * 3, [8] * 3, [0.0] * 3, [h] * 3)
    rng = np.random.default_rng(5)
    u0 = with_ghosts(rng.standard_normal((8, 8, 8, 8)), 1)
    a, b = orc.State(g, [1]), orc.State(g, [1])
    a.set(0, u0)
    b.set(0, u0)
    a.heat_run(0, kappa, 0.0, dt, 100, 1)
    b.heat_run(0, kappa, 0.0, dt, 100, 4)
    assert np.array_equal(a.interior(0), b.interior(0))


# ---------------------------------------------------------------- Model C --
def _model_c(orc, noise, steps, threads=1):
    # tests/model_c.rs:26-67: 64^2 as 2x2 blocks, h = 0.4, classic, seed 7,
    # corner seed at (H, H) radius 10 H, u0 = 0.7
    g = orc.Grid([64, 64], [32, 32], [0.0, 0.0], [H, H])
    st = orc.State(g, [1, 1])
    st.initialize_grains([(H, H, 10.0 * H)], 0.7)
    p = orc.modelc_params(noise=noise)
    dt = 0.2 * (H * H) / p.d_thermal
    st.modelc_run(p, 0.0, dt, 7, steps, wiener=True, threads=threads)
    return st.interior(0), st.interior(1)


def test_dendrite_grows_and_stays_physical(orc):
    # tests/model_c.rs:70-101
    phi0, _ = _model_c(orc, 0.0, 0)
    phi, u = _model_c(orc, 0.0, 1200)
    assert 0.95 < phi.max() < 1.1
    assert -1.1 < phi.min() < -0.95
    f0 = (phi0 > 0).mean()
    f1 = (phi > 0).mean()
    assert f1 > 1.5 * f0
    assert -0.4 < u.max() < 0.05
    assert u.min() >= -0.75


def test_stochastic_run_is_thread_count_independent(orc):
    # tests/model_c.rs:103-109 (b = 0.05, 300 steps)
    a = _model_c(orc, 0.05, 300, threads=1)
    b = _model_c(orc, 0.05, 300, threads=4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_noise_changes_the_trajectory(orc):
    # tests/model_c.rs:111-116
    quiet, _ = _model_c(orc, 0.0, 100)
    noisy, _ = _model_c(orc, 0.05, 100)
    assert not np.array_equal(quiet, noisy)
