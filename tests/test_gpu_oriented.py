"""Multi-grain (oriented) Model C on the GPU.

* FP64: bit-identical to the oracle's restatement of the reference's
  apply_oriented path without noise (several grains and orientations; block
  widths 32, 126 and a generic one; graph replay), within 1e-12 with noise.
* theta0 = 0 reproduces the axis-aligned device step bit for bit, noise
  included (the reference's zero_orientation_is_bitwise_identical pin).
* theta0 stays in both step buffers; the rotated-grain pin of the reference
  holds on the device; FP32 tracks the FP64 oracle.
"""
import math

import numpy as np
import pytest

import legendre_b200 as L
from test_oracle_oriented import arm_length
from util import centers

pytestmark = pytest.mark.gpu

H = 0.4
GRAINS = [(6.0, 7.0, 3.0, 0.3), (17.0, 20.0, 2.5, -0.7), (20.0, 6.0, 2.0, 1.2)]


def oriented_pair(sched, orc, cells, block, grains, noise, steps, seed=7, graph=False, dtype="f64"):
    grid = L.CartesianGrid(cells, block, [0.0, 0.0], [H, H])
    model = L.ModelC(0.06, 3.19, noise).with_orientations()
    sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(seed), sched, L.CudaAllocator(dtype))
    og = orc.Grid(cells, block, [0.0, 0.0], [H, H])
    os_ = orc.State(og, [1, 1, 0])
    os_.initialize_grains([g[:3] for g in grains], 0.7)
    os_.initialize_orientations(2, grains)
    if dtype == "f64":
        model.initialize_grains(grid, sim.state, [L.Grain((g[0], g[1]), g[2], g[3]) for g in grains], 0.7)
        for f in (0, 1, 2):
            assert np.array_equal(sim.state.interior(f), os_.interior(f)), f
    else:
        for f in (0, 1, 2):
            sim.state.upload(f, os_.get(f).astype(np.float32))
        model.set_orientations(sim.state)
    dt = model.stable_dt(grid.spacing)
    if steps:
        sim.run(dt, steps, graph=graph)
    p = orc.modelc_params(eps4=0.06, lam=3.19, noise=noise)
    os_.modelc_run_oriented(p, 2, 0.0, dt, seed, steps, True, threads=4)
    return sim, os_


@pytest.mark.parametrize("cells,block,graph", [
    ([64, 64], [32, 32], False),
    ([64, 64], [32, 32], True),
    ([126, 80], [126, 40], False),
    ([96, 60], [48, 20], False),
])
def test_oriented_noise_free_bit_identical_to_oracle(sched, orc, cells, block, graph):
    sim, os_ = oriented_pair(sched, orc, cells, block, GRAINS, 0.0, 120, graph=graph)
    assert np.array_equal(sim.state.interior("phi"), os_.interior(0))
    assert np.array_equal(sim.state.interior("u"), os_.interior(1))
    assert np.array_equal(sim.state.interior("theta0"), os_.interior(2))


def test_oriented_noisy_matches_oracle(sched, orc):
    sim, os_ = oriented_pair(sched, orc, [64, 64], [32, 32], GRAINS, 0.05, 200)
    assert np.allclose(sim.state.interior("phi"), os_.interior(0), rtol=1e-12, atol=1e-12)
    assert np.allclose(sim.state.interior("u"), os_.interior(1), rtol=1e-12, atol=1e-12)


def test_zero_orientation_equals_the_axis_aligned_step(sched):
    n = 64
    grid = L.CartesianGrid([n, n], [n // 2, n // 2], [0.0, 0.0], [H, H])
    out = []
    for orient in (False, True):
        model = L.ModelC(0.06, 3.19, 0.03)
        if orient:
            model.with_orientations()
        sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(7), sched, L.CudaAllocator("f64"))
        model.initialize_grains(grid, sim.state, [L.Grain((H, H), 10 * H, 0.0)], 0.7)
        sim.run(model.stable_dt(grid.spacing), 300, graph=True)
        out.append((sim.state.interior("phi"), sim.state.interior("u")))
        if orient:
            assert np.all(sim.state.interior("theta0") == 0.0)
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_theta0_stays_in_both_buffers(sched, orc):
    sim, os_ = oriented_pair(sched, orc, [64, 64], [32, 32], GRAINS, 0.0, 1)
    th = os_.interior(2)
    for _ in range(3):
        assert np.array_equal(sim.state.interior("theta0"), th)
        sim.run(0.01, 1)


def test_rotated_grain_grows_along_rotated_axes_on_the_device(sched):
    m = 96
    grid = L.CartesianGrid([m, m], [m // 2, m // 2], [0.0, 0.0], [H, H])
    c = m * H / 2.0
    x = centers([m, m], [m // 2, m // 2], [0.0, 0.0], [H, H], 0)
    y = centers([m, m], [m // 2, m // 2], [0.0, 0.0], [H, H], 1)
    wedge = math.radians(12.0)
    axes = [0.0, math.pi / 2, math.pi, -math.pi / 2]
    diags = [math.pi / 4, 3 * math.pi / 4, -math.pi / 4, -3 * math.pi / 4]
    arms = {}
    for theta0 in (0.0, math.pi / 4):
        model = L.ModelC(0.06, 3.19, 0.0).with_orientations()
        sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(7), sched, L.CudaAllocator("f64"))
        model.initialize_grains(grid, sim.state, [L.Grain((c, c), 10 * H, theta0)], 0.7)
        sim.run(model.stable_dt(grid.spacing), 700, graph=True)
        solid = sim.state.interior("phi") > 0.0
        dx, dy = x[solid] - c, y[solid] - c
        s = (np.arctan2(dy, dx), np.hypot(dx, dy))
        arms[theta0] = (arm_length(s, axes, wedge), arm_length(s, diags, wedge))
    assert arms[0.0][0] > 1.02 * arms[0.0][1]
    assert arms[math.pi / 4][1] > 1.02 * arms[math.pi / 4][0]


def test_oriented_fp32_tracks_the_fp64_oracle(sched, orc):
    sim, os_ = oriented_pair(sched, orc, [64, 64], [32, 32], GRAINS, 0.0, 300, dtype="f32")
    phi = sim.state.interior("phi").astype(np.float64)
    ref = os_.interior(0)
    assert np.sqrt(np.mean((phi - ref) ** 2)) < 1e-4
    assert np.max(np.abs(phi - ref)) < 1e-3


def _f32_sim(sched, orc, cells, block, oriented):
    grid = L.CartesianGrid(cells, block, [0.0, 0.0], [H, H])
    model = L.ModelC(0.06, 3.19, 0.05)
    if oriented:
        model = model.with_orientations()
    sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(5), sched, L.CudaAllocator("f32"))
    og = orc.Grid(cells, block, [0.0, 0.0], [H, H])
    os_ = orc.State(og, [1, 1, 0] if oriented else [1, 1])
    os_.initialize_grains([g[:3] for g in GRAINS], 0.7)
    if oriented:
        os_.initialize_orientations(2, GRAINS)
    for f in range(3 if oriented else 2):
        sim.state.upload(f, os_.get(f).astype(np.float32))
    if oriented:
        model.set_orientations(sim.state)
    return sim, model, grid


@pytest.mark.parametrize("oriented,variant", [(False, 5 + 1000 * 32), (False, 2 + 1000 * 32),
                                              (True, 5 + 1000 * 32)])
def test_fp32_runs_repeat_bit_for_bit(sched, orc, oriented, variant):
    """FP32 (contraction allowed) with noise on 40-row blocks in 32-row
    units, so each block's last unit overlaps the one below it: two runs
    from the same state give the same bits, paired or single rows, because
    every cell is stored by the one unit that owns it (two warps computing a
    row with differently contracted arithmetic could otherwise store
    different values)."""
    outs = []
    for _ in range(2):
        sim, model, grid = _f32_sim(sched, orc, [252, 80], [126, 40], oriented)
        sim.run(model.stable_dt(grid.spacing), 40, variant=variant)
        outs.append([sim.state.download(f) for f in ("phi", "u")])
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
