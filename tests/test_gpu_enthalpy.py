"""The FP64 field reduction (lg_state_field_sum) and Model C's enthalpy on a GPU.

* The device sum of a field's interior cells equals the exactly rounded sum
  (math.fsum) to within the rounding of an FP64 summation, for FP64 and FP32
  states, 2-D and 3-D, ghost widths 0, 1 and 2; it is the same bits on every
  call.
* Model C without noise conserves h^2 sum(u - phi/2) (du/dt = D lap u +
  dphi/dt / 2, phasefield.rs:411-421) to rounding, with zero-flux and with
  periodic boundaries: FP64 to 1e-12 and FP32 to 1e-6 of the enthalpy's
  scale.  With noise it moves (the noise enters phi alone).
"""
import math

import numpy as np
import pytest

import legendre_b200 as L
from util import with_ghosts

pytestmark = pytest.mark.gpu

H = 0.4


def exact_sum(state, f):
    return math.fsum(state.interior(f).astype(np.float64).reshape(-1).tolist())


def abs_sum(state, f):
    return float(np.sum(np.abs(state.interior(f).astype(np.float64))))


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("cells, block, ghosts", [
    ((64, 96), (32, 32), [1, 1, 0]),
    ((40, 24), (8, 12), [2, 0, 1]),
    ((12, 8, 16), (4, 4, 8), [1, 0, 2]),
    ((7, 5), (7, 5), [1, 1, 1]),
])
def test_field_sum_equals_the_exact_sum(sched, dtype, cells, block, ghosts):
    D = len(cells)
    grid = L.CartesianGrid(list(cells), list(block), [0.0] * D, [H] * D)
    alloc = L.CudaAllocator(dtype)
    specs = [L.FieldSpec(f"f{k}", g) for k, g in enumerate(ghosts)]
    st = L.DeviceState(grid, sched, alloc, specs)
    rng = np.random.default_rng(11 + D)
    for k, g in enumerate(ghosts):
        x = rng.standard_normal((grid.num_blocks(),) + tuple(reversed(block))) + 0.25 * k
        st.upload(f"f{k}", with_ghosts(x, g).astype(alloc.numpy_dtype))
    for k in range(len(ghosts)):
        s = st.field_sum(f"f{k}")
        assert abs(s - exact_sum(st, f"f{k}")) <= 1e-13 * abs_sum(st, f"f{k}")
        assert st.field_sum(f"f{k}") == s  # the same bits on every call


def modelc_sim(sched, dtype, noise, periodic=False, cells=(64, 96), block=(32, 32), seed=3):
    grid = L.CartesianGrid(list(cells), list(block), [0.0, 0.0], [H, H])
    if periodic:
        grid = grid.with_periodic([True, True])
    model = L.ModelC(0.05, 3.19, noise)
    model.d_thermal = 2.0
    sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(seed), sched, L.CudaAllocator(dtype))
    init = sim if dtype == "f64" else L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(seed), sched,
                                                   L.CudaAllocator("f64"))
    model.initialize_grains(grid, init.state, [L.Grain((cells[0] * H / 2, cells[1] * H / 2), 6.0)], 0.55)
    if init is not sim:  # FP32: a cast copy of the FP64 initial state
        for f in ("phi", "u"):
            sim.state.upload(f, init.state.download(f).astype(np.float32))
    return sim, grid, model


def scale(sim):
    return H * H * (abs_sum(sim.state, "u") + 0.5 * abs_sum(sim.state, "phi"))


@pytest.mark.parametrize("dtype, tol", [("f64", 1e-12), ("f32", 1e-6)])
@pytest.mark.parametrize("periodic", [False, True])
def test_modelc_conserves_enthalpy_without_noise(sched, dtype, tol, periodic):
    sim, grid, model = modelc_sim(sched, dtype, 0.0, periodic)
    h0 = model.enthalpy(grid, sim.state)
    assert h0 == pytest.approx(H * H * (exact_sum(sim.state, "u") - 0.5 * exact_sum(sim.state, "phi")),
                               rel=0, abs=1e-12 * scale(sim))
    phi0 = sim.state.interior("phi").astype(np.float64)
    sim.run(0.01, 200, graph=True)
    assert not np.array_equal(sim.state.interior("phi").astype(np.float64), phi0)  # the grain did grow
    assert abs(model.enthalpy(grid, sim.state) - h0) <= tol * scale(sim)


def test_noise_moves_the_enthalpy(sched):
    sim, grid, model = modelc_sim(sched, "f64", 0.02)
    h0 = model.enthalpy(grid, sim.state)
    sim.run(0.01, 50, graph=True)
    assert abs(model.enthalpy(grid, sim.state) - h0) > 1e-7 * scale(sim)
