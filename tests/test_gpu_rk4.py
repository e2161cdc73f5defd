"""RungeKutta4 on the GPU against the oracle's restatement of rk4.rs.

* Heat (2-D zero-flux, 3-D periodic) and Model C (axis-aligned and
  multi-grain, several block widths, graph replay): FP64 bit-identical.
* The reference's eigenmode pin (tests/heat.rs:156-168) on the device.
* FP32 Model C RK4 tracks the FP64 oracle; noise is refused.
"""
import math

import numpy as np
import pytest

import legendre_b200 as L
from util import centers, relative_eq, with_ghosts

pytestmark = pytest.mark.gpu

H = 0.4


@pytest.mark.parametrize("cells,block,periodic", [([32, 32], [8, 8], [False, False]),
                                                  ([12, 8, 16], [4, 4, 8], [True, False, True])])
def test_heat_rk4_bit_identical_to_oracle(sched, orc, cells, block, periodic):
    D = len(cells)
    h, kappa = 0.1, 0.7
    grid = L.CartesianGrid(cells, block, [0.0] * D, [h] * D).with_periodic(periodic)
    sim = L.Simulation(grid, L.FiniteDifference(), L.Heat(kappa), L.RungeKutta4(), sched, L.CudaAllocator("f64"))
    rng = np.random.default_rng(3)
    u0 = with_ghosts(rng.standard_normal((grid.num_blocks(),) + tuple(reversed(block))), 1)
    sim.state.upload("u", u0)
    dt = 0.2 * h * h / kappa
    sim.run(dt, 41, graph=True)
    og = orc.Grid(cells, block, [0.0] * D, [h] * D, periodic)
    os_ = orc.State(og, [1])
    os_.set(0, u0)
    os_.heat_run_rk4(0, kappa, 0.0, dt, 41)
    assert np.array_equal(sim.state.interior("u"), os_.interior(0))


def test_heat_rk4_matches_discrete_eigenmode_decay(sched):
    n, h, kappa, steps = 32, 0.1, 0.7, 200
    cells, block = [n, n], [n // 4, n // 4]
    grid = L.CartesianGrid(cells, block, [0.0, 0.0], [h, h])
    sim = L.Simulation(grid, L.FiniteDifference(), L.Heat(kappa), L.RungeKutta4(), sched, L.CudaAllocator("f64"))
    kx = math.pi / (n * h)
    x = centers(cells, block, [0.0, 0.0], [h, h], 0)
    sim.state.upload("u", with_ghosts(np.cos(kx * x), 1))
    dt = 0.25 * h * h / kappa
    sim.run(dt, steps)
    z = dt * kappa * (2.0 - 2.0 * math.cos(kx * h)) / (h * h)
    factor = (1.0 - z + z * z / 2.0 - z ** 3 / 6.0 + z ** 4 / 24.0) ** steps
    assert np.all(relative_eq(sim.state.interior("u"), factor * np.cos(kx * x), 1e-10, 1e-12))


GRAINS = [(6.0, 7.0, 3.0, 0.3), (17.0, 20.0, 2.5, -0.7)]


@pytest.mark.parametrize("orient", [False, True])
@pytest.mark.parametrize("cells,block,graph", [([64, 64], [32, 32], True), ([96, 60], [48, 20], False),
                                               ([14, 6], [7, 3], False)])
def test_modelc_rk4_bit_identical_to_oracle(sched, orc, orient, cells, block, graph):
    grid = L.CartesianGrid(cells, block, [0.0, 0.0], [H, H])
    model = L.ModelC(0.06, 3.19, 0.0)
    if orient:
        model.with_orientations()
    sim = L.Simulation(grid, L.FiniteVolume(), model, L.RungeKutta4(), sched, L.CudaAllocator("f64"))
    grains = [(g[0] * cells[0] / 64, g[1] * cells[1] / 64, g[2] * min(cells) / 64, g[3]) for g in GRAINS]
    model.initialize_grains(grid, sim.state, [L.Grain((g[0], g[1]), g[2], g[3] if orient else 0.0) for g in grains],
                            0.7)
    og = orc.Grid(cells, block, [0.0, 0.0], [H, H])
    os_ = orc.State(og, [1, 1, 0] if orient else [1, 1])
    os_.initialize_grains([g[:3] for g in grains], 0.7)
    if orient:
        os_.initialize_orientations(2, grains)
    dt = model.stable_dt(grid.spacing)
    sim.run(dt, 60, graph=graph)
    p = orc.modelc_params(eps4=0.06, lam=3.19)
    os_.modelc_run_rk4(p, 0.0, dt, 60, theta_field=2 if orient else -1, threads=4)
    assert np.array_equal(sim.state.interior("phi"), os_.interior(0))
    assert np.array_equal(sim.state.interior("u"), os_.interior(1))
    assert sim.time() == pytest.approx(60 * dt) and sim.step_index() == 60


def test_modelc_rk4_fp32_tracks_the_fp64_oracle(sched, orc):
    cells, block = [64, 64], [32, 32]
    grid = L.CartesianGrid(cells, block, [0.0, 0.0], [H, H])
    model = L.ModelC(0.06, 3.19, 0.0)
    sim = L.Simulation(grid, L.FiniteVolume(), model, L.RungeKutta4(), sched, L.CudaAllocator("f32"))
    og = orc.Grid(cells, block, [0.0, 0.0], [H, H])
    os_ = orc.State(og, [1, 1])
    os_.initialize_grains([(H, H, 10 * H)], 0.7)
    sim.state.upload("phi", os_.get(0).astype(np.float32))
    sim.state.upload("u", os_.get(1).astype(np.float32))
    dt = model.stable_dt(grid.spacing)
    sim.run(dt, 200, graph=True)
    os_.modelc_run_rk4(orc.modelc_params(eps4=0.06, lam=3.19), 0.0, dt, 200, threads=4)
    phi = sim.state.interior("phi").astype(np.float64)
    assert np.sqrt(np.mean((phi - os_.interior(0)) ** 2)) < 1e-4
    assert np.max(np.abs(phi - os_.interior(0))) < 1e-3


def test_rk4_refuses_noise(sched):
    grid = L.CartesianGrid([32, 32], [16, 16], [0.0, 0.0], [H, H])
    with pytest.raises(TypeError):
        L.Simulation(grid, L.FiniteVolume(), L.ModelC(0.06, 3.19, 0.01), L.RungeKutta4(), sched,
                     L.CudaAllocator("f64"))
