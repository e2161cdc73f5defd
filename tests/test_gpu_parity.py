"""CUDA path against the oracle on the same seeded inputs (needs a GPU).

FP64 results are compared bit for bit; the noisy Model C path compares the
integer key stream exactly and the Gaussian within 1e-12 relative.
"""
import math

import numpy as np
import pytest

import legendre_b200 as L
from util import centers, relative_eq, with_ghosts

pytestmark = pytest.mark.gpu

H = 0.4


def dev_state(sched, cells, block, ghosts, periodic=None, spacing=1.0, dtype="f64"):
    D = len(cells)
    grid = L.CartesianGrid(cells, block, [0.0] * D, [spacing] * D).with_periodic(periodic or [False] * D)
    specs = [L.FieldSpec(f"f{i}", g) for i, g in enumerate(ghosts)]
    return L.DeviceState(grid, sched, L.CudaAllocator(dtype), specs)


HALO_CASES = [
    ([8], [4], 1, None),
    ([8], [4], 2, None),
    ([8], [4], 1, [True]),
    ([4], [4], 2, [True]),
    ([4, 4], [4, 4], 1, [True, False]),
    ([12, 8], [4, 4], 1, [True, False]),
    ([8, 12], [4, 4], 2, [False, True]),
    ([64, 64], [32, 32], 1, None),
    ([16, 16, 16], [8, 8, 8], 1, None),
    ([12, 12, 12], [6, 4, 3], 1, [True, False, True]),
    ([12, 12, 12], [6, 4, 3], 3, [False, True, True]),
    ([6, 6, 6], [6, 6, 6], 2, [True, True, True]),
]


@pytest.mark.parametrize("cells,block,ghost,periodic", HALO_CASES)
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_halo_fill_matches_oracle(sched, orc, cells, block, ghost, periodic, dtype):
    D = len(cells)
    st = dev_state(sched, cells, block, [ghost], periodic, dtype=dtype)
    og = orc.Grid(cells, block, [0.0] * D, [1.0] * D, periodic)
    os_ = orc.State(og, [ghost])
    rng = np.random.default_rng(sum(cells) + ghost)
    data = rng.standard_normal((og.num_blocks(),) + og.slab_shape(ghost))
    if dtype == "f32":
        data = data.astype(np.float32).astype(np.float64)
    st.upload(0, data)
    os_.set(0, data)
    st.fill_ghosts(0)
    os_.fill_ghosts(0)
    assert np.array_equal(st.download(0).astype(np.float64), os_.get(0))


def _heat_pair(sched, orc, cells, block, periodic, h, kappa, dt, steps, graph=False, seed=3):
    D = len(cells)
    grid = L.CartesianGrid(cells, block, [0.0] * D, [h] * D).with_periodic(periodic or [False] * D)
    model = L.Heat(kappa)
    sim = L.Simulation(grid, L.FiniteDifference(), model, L.ForwardEuler(), sched, L.CudaAllocator("f64"))
    rng = np.random.default_rng(seed)
    u0 = with_ghosts(rng.standard_normal((grid.num_blocks(),) + tuple(reversed(block))), 1)
    sim.state.upload("u", u0)
    sim.run(dt, steps, graph=graph)
    og = orc.Grid(cells, block, [0.0] * D, [h] * D, periodic)
    os_ = orc.State(og, [1])
    os_.set(0, u0)
    t = os_.heat_run(0, kappa, 0.0, dt, steps)
    return sim, os_, t


@pytest.mark.parametrize("cells,block,periodic", [
    ([16, 16, 16], [8, 8, 8], None),
    ([32, 32], [16, 16], [True, True]),
    ([32, 32], [32, 32], [True, True]),
    ([64], [16], [True]),
    ([24, 16, 8], [8, 8, 4], [False, True, False]),
    ([12, 8, 16], [12, 4, 8], [True, True, True]),   # one block along x: the periodic halo is the block itself
    ([8, 8, 40], [8, 8, 40], [False, False, True]),  # one block of 40 planes, split into z-ranges
    ([9, 10, 12], [3, 5, 6], [True, False, False]),   # odd block width: the cp.async-staged form
    ([32, 48, 48], [16, 16, 16], [False, True, False]),  # 16^3 blocks, tensor-copy staged, whole blocks per CTA
    # the tensor-copy form on 64 and 512 blocks of 16^3 and on 64 blocks split into z-ranges
    ([64, 64, 64], [16, 16, 16], [True, True, True]),
    ([64, 64, 64], [16, 16, 16], None),
    ([128, 128, 128], [16, 16, 16], [True, False, True]),
    ([32, 32, 160], [8, 8, 40], [False, True, True]),
])
def test_heat_bit_identical_to_oracle(sched, orc, cells, block, periodic):
    sim, os_, t = _heat_pair(sched, orc, cells, block, periodic, 0.1, 0.7, 0.5 / 6.0 * 0.01 / 0.7, 37)
    assert np.array_equal(sim.state.interior("u"), os_.interior(0))
    assert sim.time() == t and sim.step_index() == 37


def test_heat_graph_replay_identical(sched, orc):
    sim, os_, _ = _heat_pair(sched, orc, [16, 16, 16], [8, 8, 8], None, 0.1, 0.7, 0.001, 131, graph=True)
    assert np.array_equal(sim.state.interior("u"), os_.interior(0))


def test_heat_benchmark_config_short(sched, orc):
    # 96^3 periodic, 6^3 blocks of 16^3, dt = 0.15 h^2, sine + seeded noise IC
    h = 1.0 / 96
    grid = L.CartesianGrid([96] * 3, [16] * 3, [0.0] * 3, [h] * 3).with_periodic([True] * 3)
    model = L.Heat(1.0)
    sim = L.Simulation(grid, L.FiniteDifference(), model, L.ForwardEuler(), sched, L.CudaAllocator("f64"))
    model.initialize_sine_noise(sim.state, 42, 1e-3)
    u0 = sim.state.download("u")
    # the initial condition against its definition
    x, y, z = (centers([96] * 3, [16] * 3, [0.0] * 3, [h] * 3, d) for d in range(3))
    ref = np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * np.sin(2 * np.pi * z)
    assert np.max(np.abs(sim.state.interior("u") - ref)) <= 1e-3 + 1e-14
    dt = 0.15 * h * h
    sim.run(dt, 20, graph=True)
    og = orc.Grid([96] * 3, [16] * 3, [0.0] * 3, [h] * 3, [True] * 3)
    os_ = orc.State(og, [1])
    os_.set(0, u0)
    os_.heat_run(0, 1.0, 0.0, dt, 20, 8)
    assert np.array_equal(sim.state.interior("u"), os_.interior(0))


def test_heat_analytic_decay_on_gpu(sched):
    # tests/heat3d.rs:82-137 on the device
    h, kappa, n = 0.1, 0.7, 16
    grid = L.CartesianGrid([n] * 3, [n // 2] * 3, [0.0] * 3, [h] * 3)
    model = L.Heat(kappa)
    sim = L.Simulation(grid, L.FiniteDifference(), model, L.ForwardEuler(), sched, L.CudaAllocator("f64"))
    kx = math.pi / (n * h)
    x = centers([n] * 3, [n // 2] * 3, [0.0] * 3, [h] * 3, 0)
    u0 = np.vectorize(math.cos)(kx * x)
    sim.state.upload("u", with_ghosts(u0, 1))
    dt = sim.stable_dt()
    sim.run(dt, 200)
    lam = (2.0 - 2.0 * math.cos(kx * h)) / (h * h)
    assert relative_eq(sim.state.interior("u"), (1.0 - dt * kappa * lam) ** 200 * u0, 1e-10, 1e-12).all()


# ---------------------------------------------------------------- Model C --
def _modelc_pair(sched, orc, cells, block, grains, noise, steps, seed=7, graph=False, dtype="f64", eps4=0.06,
                 lam=3.19, threads=4):
    grid = L.CartesianGrid(cells, block, [0.0, 0.0], [H, H])
    model = L.ModelC(eps4, lam, noise)
    sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(seed), sched, L.CudaAllocator(dtype))
    og = orc.Grid(cells, block, [0.0, 0.0], [H, H])
    os_ = orc.State(og, [1, 1])
    os_.initialize_grains([(g[0], g[1], g[2]) for g in grains], 0.7)
    if dtype == "f64":
        model.initialize_grains(grid, sim.state, [L.Grain((g[0], g[1]), g[2]) for g in grains], 0.7)
        assert np.array_equal(sim.state.interior("phi"), os_.interior(0))
        assert np.array_equal(sim.state.interior("u"), os_.interior(1))
    else:
        sim.state.upload("phi", os_.get(0))
        sim.state.upload("u", os_.get(1))
    dt = model.stable_dt(grid.spacing)
    if steps:
        sim.run(dt, steps, graph=graph)
    p = orc.modelc_params(eps4=eps4, lam=lam, noise=noise)
    t = os_.modelc_run(p, 0.0, dt, seed, steps, wiener=True, threads=threads)
    return sim, os_, t


@pytest.mark.parametrize("cells,block,grains", [
    ([64, 64], [32, 32], [(H, H, 10 * H)]),
    ([64, 64], [64, 64], [(H, H, 10 * H)]),
    ([96, 64], [32, 32], [(10.0, 12.0, 4.0), (30.0, 14.0, 3.0)]),
    ([48, 80], [16, 16], [(9.5, 16.0, 5.0)]),
])
def test_modelc_noise_free_bit_identical(sched, orc, cells, block, grains):
    sim, os_, t = _modelc_pair(sched, orc, cells, block, grains, 0.0, 300)
    assert np.array_equal(sim.state.interior("phi"), os_.interior(0))
    assert np.array_equal(sim.state.interior("u"), os_.interior(1))
    assert sim.time() == t


def test_modelc_decomposition_independent_without_noise(sched, orc):
    res = []
    for block in ([64, 64], [32, 32], [16, 16]):
        sim, _, _ = _modelc_pair(sched, orc, [64, 64], block, [(H, H, 10 * H)], 0.0, 50)
        phi = sim.state.interior("phi")
        nb = 64 // block[0]
        full = phi.reshape(nb, nb, block[1], block[0]).transpose(0, 2, 1, 3).reshape(64, 64)
        res.append(full)
    assert np.array_equal(res[0], res[1]) and np.array_equal(res[0], res[2])


def test_standard_normal_within_1e12(sched, orc):
    rng = np.random.default_rng(11)
    keys = rng.integers(0, 2**63, size=100_000, dtype=np.int64).astype(np.uint64) * np.uint64(2) + np.uint64(1)
    keys[:4] = [0, 1, 2**64 - 1, 0xD1B54A32D192ED03]
    import ctypes as C
    out = np.empty(keys.size)
    L._native.check(L._native.lib.lg_standard_normal(sched.handle, keys.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                     keys.size, out.ctypes.data_as(C.POINTER(C.c_double))),
                    sched.handle)
    ref = orc.standard_normal(keys)
    assert np.all(np.abs(out - ref) <= 1e-12 * np.abs(ref))


def test_modelc_noisy_matches_oracle(sched, orc):
    sim, os_, t = _modelc_pair(sched, orc, [64, 64], [32, 32], [(H, H, 10 * H)], 0.05, 300)
    phi, phi_ref = sim.state.interior("phi"), os_.interior(0)
    assert np.allclose(phi, phi_ref, rtol=1e-12, atol=1e-12)
    assert np.allclose(sim.state.interior("u"), os_.interior(1), rtol=1e-12, atol=1e-12)
    # the noise must actually be there
    quiet, _, _ = _modelc_pair(sched, orc, [64, 64], [32, 32], [(H, H, 10 * H)], 0.0, 300)
    assert not np.allclose(phi, quiet.state.interior("phi"), atol=1e-6)


def test_modelc_graph_replay_identical(sched, orc):
    a, os_, _ = _modelc_pair(sched, orc, [64, 64], [32, 32], [(H, H, 10 * H)], 0.05, 150, graph=True)
    b, _, _ = _modelc_pair(sched, orc, [64, 64], [32, 32], [(H, H, 10 * H)], 0.05, 150, graph=False)
    assert np.array_equal(a.state.interior("phi"), b.state.interior("phi"))
    assert np.array_equal(a.state.interior("u"), b.state.interior("u"))


def test_modelc_fp32_error_against_fp64_oracle(sched, orc):
    sim, os_, _ = _modelc_pair(sched, orc, [64, 64], [32, 32], [(H, H, 10 * H)], 0.0, 400, dtype="f32")
    phi = sim.state.interior("phi").astype(np.float64)
    ref = os_.interior(0)
    l2 = np.sqrt(np.mean((phi - ref) ** 2))
    assert l2 < 1e-4, l2
    assert np.max(np.abs(phi - ref)) < 1e-3


def test_dendrite_grows_and_stays_physical_on_gpu(sched, orc):
    # tests/model_c.rs:70-101 on the device
    sim, _, _ = _modelc_pair(sched, orc, [64, 64], [32, 32], [(H, H, 10 * H)], 0.0, 0)
    phi0 = sim.state.interior("phi")
    dt = sim.model.stable_dt(sim.grid.spacing)
    sim.run(dt, 1200, graph=True)
    phi, u = sim.state.interior("phi"), sim.state.interior("u")
    assert 0.95 < phi.max() < 1.1 and -1.1 < phi.min() < -0.95
    assert (phi > 0).mean() > 1.5 * (phi0 > 0).mean()
    assert -0.4 < u.max() < 0.05 and u.min() >= -0.75


@pytest.mark.parametrize("variant", [1, 2, 2 + 1000 * 16, 2 + 1000 * 24, 2 + 1000 * 7, 2 + 1000 * 5000,
                                     5, 5 + 1000 * 8, 6 + 1000 * 16, 7 + 1000 * 32, 12, 13 + 1000 * 8,
                                     15 + 1000 * 16, 17 + 1000 * 32])
@pytest.mark.parametrize("noise", [0.0, 0.05])
def test_modelc_kernel_variants_bit_identical(sched, orc, variant, noise):
    # every kernel shape (reference order, column tiles of any height) gives
    # the same bits; without noise they equal the oracle's
    cells, block = [96, 64], [32, 32]
    grains = [(10.0, 12.0, 4.0), (30.0, 14.0, 3.0)]
    grid = L.CartesianGrid(cells, block, [0.0, 0.0], [H, H])
    model = L.ModelC(0.06, 3.19, noise)
    sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(3), sched, L.CudaAllocator("f64"))
    model.initialize_grains(grid, sim.state, [L.Grain((g[0], g[1]), g[2]) for g in grains], 0.7)
    sim.run(model.stable_dt(grid.spacing), 40, variant=variant)
    ref = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(3), sched, L.CudaAllocator("f64"))
    model.initialize_grains(grid, ref.state, [L.Grain((g[0], g[1]), g[2]) for g in grains], 0.7)
    ref.run(model.stable_dt(grid.spacing), 40, variant=1)
    assert np.array_equal(sim.state.download("phi"), ref.state.download("phi"))
    assert np.array_equal(sim.state.download("u"), ref.state.download("u"))


@pytest.mark.parametrize("block", [[7, 5], [1, 3], [33, 20], [256, 8]])
def test_modelc_tile_ragged_blocks(sched, orc, block):
    cells = [block[0] * 3, block[1] * 2]
    g = (cells[0] * H / 2, cells[1] * H / 2, 2.0)
    sim, os_, _ = _modelc_pair(sched, orc, cells, block, [g], 0.0, 25)
    assert np.array_equal(sim.state.interior("phi"), os_.interior(0))
    assert np.array_equal(sim.state.interior("u"), os_.interior(1))


@pytest.mark.parametrize("block", [[33, 20], [126, 6], [126, 40], [7, 3]])
@pytest.mark.parametrize("paired", [2, 5, 15])
def test_modelc_tile_ragged_blocks_noisy(sched, orc, block, paired):
    # strips whose last lanes lie past the block edge: with noise, the strip
    # kernel gives the bits of the one-thread-per-cell kernel
    cells = [block[0] * 2, block[1] * 2]
    grid = L.CartesianGrid(cells, block, [0.0, 0.0], [H, H])
    model = L.ModelC(0.06, 3.19, 0.05)
    sims = []
    for variant in (paired, 1):
        sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(5), sched, L.CudaAllocator("f64"))
        model.initialize_grains(grid, sim.state, [L.Grain((cells[0] * H / 2, cells[1] * H / 2), 2.0)], 0.7)
        sim.run(model.stable_dt(grid.spacing), 30, variant=variant)
        sims.append(sim)
    for f in ("phi", "u"):
        assert np.array_equal(sims[0].state.download(f), sims[1].state.download(f))


def test_modelc_fp32_noisy_tracks_fp64_oracle(sched, orc):
    # same counter-based noise realization in both precisions
    sim, os_, _ = _modelc_pair(sched, orc, [64, 64], [32, 32], [(H, H, 10 * H)], 0.05, 300, dtype="f32")
    phi = sim.state.interior("phi").astype(np.float64)
    ref = os_.interior(0)
    assert np.sqrt(np.mean((phi - ref) ** 2)) < 1e-4
    assert np.max(np.abs(phi - ref)) < 2e-3


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_autotune_restores_the_state_and_keeps_the_results(sched, orc, dtype):
    # the tuner times every variant from a copy of the state and puts it back;
    # runs with the chosen variant give the oracle's bits (FP64, no noise)
    sim, os_, _ = _modelc_pair(sched, orc, [96, 64], [32, 32], [(10.0, 12.0, 4.0)], 0.0, 10, dtype=dtype)
    before = [sim.state.download(f).copy() for f in ("phi", "u")]
    t0, k0 = sim.time(), sim.step_index()
    dt = sim.model.stable_dt(sim.grid.spacing)
    variant, ms = sim.autotune(dt, trial_steps=5)
    assert variant % 1000 in (2, 3, 4, 5, 6, 7, 12, 13, 14, 15, 16, 17) and ms > 0.0
    for f, b in zip(("phi", "u"), before):
        assert np.array_equal(sim.state.download(f), b)
    assert sim.time() == t0 and sim.step_index() == k0
    if dtype == "f64":
        sim.run(dt, 30, graph=True)
        os_.modelc_run(orc.modelc_params(eps4=0.06, lam=3.19, noise=0.0), t0, dt, 7, 30, wiener=True, threads=4)
        assert np.array_equal(sim.state.interior("phi"), os_.interior(0))
        assert np.array_equal(sim.state.interior("u"), os_.interior(1))


@pytest.mark.parametrize("variant", [12, 15 + 1000 * 8])
def test_modelc_work_list_across_runs_and_graphs(sched, orc, variant):
    """The persistent work-list form keeps its per-step unit counters right
    across calls (odd step counts, graph replays, a call after the tuner's
    trial steps) and gives the static schedule's bits."""
    cells, block = [96, 64], [32, 32]
    grains = [(10.0, 12.0, 4.0), (30.0, 14.0, 3.0)]
    grid = L.CartesianGrid(cells, block, [0.0, 0.0], [H, H])
    model = L.ModelC(0.06, 3.19, 0.05)
    sims = []
    for v in (variant, 2):
        sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(9), sched, L.CudaAllocator("f64"))
        model.initialize_grains(grid, sim.state, [L.Grain((g[0], g[1]), g[2]) for g in grains], 0.7)
        dt = model.stable_dt(grid.spacing)
        sim.run(dt, 3, graph=True, variant=v)
        if v == variant:
            sim.autotune(dt, trial_steps=3)
        sim.run(dt, 4, graph=True, variant=v)
        sim.run(dt, 5, graph=False, variant=v)
        sims.append(sim)
    for f in ("phi", "u"):
        assert np.array_equal(sims[0].state.download(f), sims[1].state.download(f))


_M64 = (1 << 64) - 1


def _unxorshift(y, s):
    z = y
    for _ in range(64 // s + 1):
        z = y ^ (z >> s)
    return z & _M64


def _splitmix64_inverse(y):
    """The key whose SplitMix64 output is y (each step of the finalizer is a
    bijection of 64-bit words)."""
    z = _unxorshift(y, 31)
    z = (z * pow(0x94D049BB133111EB, -1, 1 << 64)) & _M64
    z = _unxorshift(z, 27)
    z = (z * pow(0xBF58476D1CE4E5B9, -1, 1 << 64)) & _M64
    z = _unxorshift(z, 30)
    return (z - 0x9E3779B97F4A7C15) & _M64


def test_standard_normal_within_1e12_at_the_hard_arguments(sched, orc):
    """Keys chosen through the inverse generator so that the radius uniform u
    sits next to 1 (ln u tiny) and the angle uniform v next to 1/4, 1/2, 3/4
    and 1 (cos(2 pi v) next to its zeros and extremes)."""
    from legendre_b200.rng import splitmix64

    assert all(splitmix64(_splitmix64_inverse(y)) == y for y in (0, 1, 2**63, _M64, 0x123456789ABCDEF))
    keys = []
    for m in range(1, 2000):  # u = 1 - m 2^-53: a's top 53 bits near all ones
        keys.append(_splitmix64_inverse(((1 << 53) - m) << 11))
    for center in (1 << 51, 1 << 52, 3 << 51, (1 << 53) - 1):  # v near 1/4, 1/2, 3/4, 1
        for d in range(-300, 300):
            b = ((center + d) % (1 << 53)) << 11
            a = _splitmix64_inverse(b) ^ 0xD1B54A32D192ED03
            keys.append(_splitmix64_inverse(a))
    keys = np.array(keys, dtype=np.uint64)
    import ctypes as C
    out = np.empty(keys.size)
    L._native.check(L._native.lib.lg_standard_normal(sched.handle, keys.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                     keys.size, out.ctypes.data_as(C.POINTER(C.c_double))),
                    sched.handle)
    ref = orc.standard_normal(keys)
    assert np.all(np.abs(out - ref) <= 1e-12 * np.abs(ref)), np.max(np.abs(out - ref) / np.abs(ref))
