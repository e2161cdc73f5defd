"""The workloads the bench times, against the oracle at their own sizes and
parameters (needs a GPU).

* Model C 4096^2 as 16x16 blocks of 256^2 (D = 2, lambda = 2/0.6267,
  eps4 = 0.05, dt = 0.008, Delta = 0.55, 16 seeded grains), with the kernel
  variant the autotuner picks for it: bit-identical without noise, within
  1e-12 with b = 0.01.
* Model C 10080^2 = 101.6M cells as 80x80 blocks of 126^2 (Delta = 0.5, 64
  grains), likewise.
* The FP32 step at 4096^2 against the FP64 oracle, the error the bench
  reports.
* Berger-Oliger AMR on a 1024^2 base of 32^2 blocks with three refined levels
  at ratio 2, |grad phi| > 0.05 tagging and a regrid every 50 coarse steps,
  through the regrids that build all four levels: bitwise.
* The batched ensemble, 256 instances of 256^2 (4x4 blocks of 64^2) with
  their own eps4, Delta and seed and b = 0.005: sampled instances against
  their own oracle runs.
* Heat 96^3 periodic as 6^3 blocks of 16^3 for its full 2000 steps:
  bitwise; heat 512^3 as 32^3 blocks of 16^3, 6 steps: bitwise.

The oracle follows src/physics/phasefield.rs:353-422 (the Model C drift),
src/core/driver.rs:117-185 (the Euler-Maruyama update),
src/geometry/amr/adapt.rs:145-237 (the regrid) and
src/integrators/subcycling.rs:63-267 (the subcycled step).
"""
import math
import os

import numpy as np
import pytest

import legendre_b200 as L

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
LAM = 2.0 / 0.6267
D_THERMAL = 2.0
EPS4 = 0.05
DT = 0.008
H = 0.4


def _uniform_pair(sched, orc, cells, block, ngrains, u0, noise, dtype="f64", seed=42):
    grid = L.CartesianGrid([cells, cells], [block, block], [0.0, 0.0], [H, H])
    model = L.ModelC(EPS4, LAM, noise)
    model.d_thermal = D_THERMAL
    sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(seed), sched, L.CudaAllocator(dtype))
    grains = L.seed_positions(cells, H, ngrains, seed, radius=8.0)
    og = orc.Grid([cells, cells], [block, block], [0.0, 0.0], [H, H])
    os_ = orc.State(og, [1, 1])
    os_.initialize_grains([(g.center[0], g.center[1], g.radius) for g in grains], u0)
    if dtype == "f64":
        model.initialize_grains(grid, sim.state, grains, u0)
        assert np.array_equal(sim.state.interior("phi"), os_.interior(0))
        assert np.array_equal(sim.state.interior("u"), os_.interior(1))
    else:
        sim.state.upload("phi", os_.get(0).astype(np.float32))
        sim.state.upload("u", os_.get(1).astype(np.float32))
    return sim, os_


def _step_both(sim, os_, orc, noise, steps, seed=42):
    variant, _ = sim.autotune(DT, trial_steps=3)
    sim.run(DT, steps, graph=True)
    p = orc.modelc_params(eps4=EPS4, lam=LAM, d_thermal=D_THERMAL, noise=noise)
    t = os_.modelc_run(p, 0.0, DT, seed, steps, wiener=True, threads=THREADS)
    return variant, t


@pytest.mark.parametrize("cells, block, ngrains, u0, steps", [
    (4096, 256, 16, 0.55, 4),
    (10080, 126, 64, 0.5, 2),
])
@pytest.mark.parametrize("noise", [0.0, 0.01])
def test_model_c_benchmark_grid_against_oracle(sched, orc, cells, block, ngrains, u0, steps, noise):
    sim, os_ = _uniform_pair(sched, orc, cells, block, ngrains, u0, noise)
    variant, t = _step_both(sim, os_, orc, noise, steps)
    assert variant % 1000 in (2, 3, 4, 5, 6, 7, 12, 13, 14, 15, 16, 17)
    for f in (0, 1):
        got, ref = sim.state.interior(("phi", "u")[f]), os_.interior(f)
        if noise == 0.0:
            assert np.array_equal(got, ref), f"field {f} differs (variant {variant})"
        else:
            assert np.allclose(got, ref, rtol=1e-12, atol=1e-12), f"field {f}: {np.max(np.abs(got - ref))}"
    assert sim.time() == t
    del sim, os_


def test_model_c_fp32_benchmark_grid_against_fp64_oracle(sched, orc):
    """The bench's FP32 error, at its own grid, against the oracle itself:
    phi L2 <= 1e-4 after 20 noisy steps."""
    sim, os_ = _uniform_pair(sched, orc, 4096, 256, 16, 0.55, 0.01, dtype="f32")
    _step_both(sim, os_, orc, 0.01, 20)
    phi = sim.state.interior("phi").astype(np.float64)
    ref = os_.interior(0)
    assert np.sqrt(np.mean((phi - ref) ** 2)) <= 1e-4
    assert np.max(np.abs(phi - ref)) <= 1e-3
    assert np.mean(phi > 0) == np.mean(ref > 0)


def test_amr_benchmark_hierarchy_across_a_regrid(sched, orc):
    """1024^2 base of 32^2 blocks, three refined levels at ratio 2, tagging
    |grad phi| > 0.05, a regrid every 50 coarse steps, one central grain of
    radius 8, Delta = 0.55, no noise: 110 subcycled coarse steps -- regrids at
    steps 0, 50 and 100 deepen the hierarchy one level each -- bitwise."""
    n, block = 1024, 32
    base = L.CartesianGrid([n, n], [block, block], [0.0, 0.0], [H, H])
    grid = L.AmrGrid.from_patches(base, [2, 2, 2], [])
    model = L.ModelC(EPS4, LAM, 0.0)
    model.d_thermal = D_THERMAL
    policy = dict(every=50, buffer=2, efficiency=0.8, min_width=4, threshold=0.05)
    adapt = L.BergerOliger(L.GradientTagger("phi", policy["threshold"]),
                           L.RegridPolicy(policy["every"], policy["buffer"], L.ClusterParams(0.8, 4)))
    dev = L.AmrSimulation(grid, L.FiniteVolume(), model, L.Subcycling(0), sched, L.CudaAllocator("f64"), adapt)
    ref = orc.AmrSim([n, n], [block, block], H, [2, 2, 2], [], model="modelc",
                     params=orc.modelc_params(eps4=EPS4, lam=LAM, d_thermal=D_THERMAL), integrator="subcycling",
                     seed=0, policy=dict(policy, field=0))
    c = n * H / 2.0
    for f, fn in ((0, lambda x, y: np.maximum(-1.0, -np.vectorize(math.tanh)(
            (np.vectorize(math.hypot)(x - c, y - c) - 8.0) / math.sqrt(2.0)))),
                  (1, lambda x, y: np.full_like(x, -0.55))):
        slabs = ref.get(f)
        for b in range(ref.num_blocks):
            xs, ys = ref.centers(b)
            slabs[b][1:-1, 1:-1] = fn(xs, ys)
        ref.set(f, slabs)
        dev.set(f, slabs)
    dt = ref.suggested_dt()
    assert dev.stable_dt() == dt
    dev.run(dt, 110, graph=True)
    ref.step(dt, 110)
    assert dev.num_levels == ref.num_levels == 4
    assert dev.epoch == ref.epoch >= 3
    assert dev.patches() == ref.patches()
    for f in (0, 1):
        for a, b in zip(dev.get(f), ref.get(f)):
            assert np.array_equal(a[1:-1, 1:-1], b[1:-1, 1:-1])


def _ensemble_inputs(ninst, n):
    from legendre_b200.rng import mix_key, unit_open

    eps4 = [0.02 + 0.05 * unit_open(mix_key(42, [i, 0])) for i in range(ninst)]
    delta = [0.45 + 0.2 * unit_open(mix_key(42, [i, 1])) for i in range(ninst)]
    seeds = [mix_key(42, [i, 2]) for i in range(ninst)]
    x = (np.arange(n) + 0.5) * H
    r = np.hypot(x[None, :] - n * H / 2, x[:, None] - n * H / 2)
    phi = np.maximum(-1.0, -np.tanh((r - 8.0) / math.sqrt(2.0)))
    return eps4, delta, seeds, phi


def _to_slabs(a, block):
    ny, nx = a.shape
    nbx, nby = nx // block, ny // block
    out = np.zeros((nbx * nby, block + 2, block + 2))
    for by in range(nby):
        for bx in range(nbx):
            out[bx + by * nbx, 1:-1, 1:-1] = a[by * block:(by + 1) * block, bx * block:(bx + 1) * block]
    return out


def _from_blocks(s, n, block):
    nb = n // block
    out = np.empty((n, n))
    for by in range(nb):
        for bx in range(nb):
            out[by * block:(by + 1) * block, bx * block:(bx + 1) * block] = s[bx + by * nb]
    return out


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_ensemble_benchmark_batch_against_oracle(sched, orc, dtype):
    """All 256 instances of 256^2 step in one launch; instances 0, 97 and 255
    each equal their own oracle run (FP64 within 1e-12 with noise; FP32
    phi L2 <= 1e-4)."""
    ninst, n, block, noise, steps = 256, 256, 64, 0.005, 20
    eps4, delta, seeds, phi = _ensemble_inputs(ninst, n)
    grid = L.CartesianGrid([n, n], [block, block], [0.0, 0.0], [H, H])
    model = L.ModelC(0.05, LAM, noise)
    model.d_thermal = D_THERMAL
    ens = L.Ensemble(grid, model, eps4, seeds, sched, dtype=dtype)
    ens.set("phi", np.broadcast_to(phi, (ninst, n, n)))
    ens.set("u", -np.asarray(delta)[:, None, None] * np.ones((1, n, n)))
    dt = 0.2 * H * H / D_THERMAL
    ens.run(dt, steps, graph=True)
    got_phi, got_u = ens.get("phi"), ens.get("u")
    og = orc.Grid([n, n], [block, block], [0.0, 0.0], [H, H])
    for i in (0, 97, 255):
        os_ = orc.State(og, [1, 1])
        os_.set(0, _to_slabs(phi, block))
        os_.set(1, _to_slabs(np.full((n, n), -delta[i]), block))
        p = orc.modelc_params(eps4=eps4[i], lam=LAM, d_thermal=D_THERMAL, noise=noise)
        os_.modelc_run(p, 0.0, dt, seeds[i], steps, wiener=True, threads=THREADS)
        rp, ru = (_from_blocks(os_.interior(f), n, block) for f in (0, 1))
        if dtype == "f64":
            assert np.allclose(got_phi[i], rp, rtol=1e-12, atol=1e-12)
            assert np.allclose(got_u[i], ru, rtol=1e-12, atol=1e-12)
        else:
            assert np.sqrt(np.mean((got_phi[i].astype(np.float64) - rp) ** 2)) <= 1e-4
    ens._destroy()


def test_heat_benchmark_config_full_run(sched, orc):
    """96^3 periodic as 6^3 blocks of 16^3, dt = 0.15 h^2, sine + seeded
    noise, all 2000 steps: bitwise."""
    h = 1.0 / 96
    grid = L.CartesianGrid([96] * 3, [16] * 3, [0.0] * 3, [h] * 3).with_periodic([True] * 3)
    model = L.Heat(1.0)
    sim = L.Simulation(grid, L.FiniteDifference(), model, L.ForwardEuler(), sched, L.CudaAllocator("f64"))
    model.initialize_sine_noise(sim.state, 42, 1e-3)
    u0 = sim.state.download("u")
    dt = 0.15 * h * h
    sim.run(dt, 2000, graph=True)
    og = orc.Grid([96] * 3, [16] * 3, [0.0] * 3, [h] * 3, [True] * 3)
    os_ = orc.State(og, [1])
    os_.set(0, u0)
    t = os_.heat_run(0, 1.0, 0.0, dt, 2000, THREADS)
    assert np.array_equal(sim.state.interior("u"), os_.interior(0))
    assert sim.time() == t


def test_heat_large_cube_against_oracle(sched, orc):
    """512^3 periodic as 32^3 blocks of 16^3 (the bench's large heat
    workload, on the tensor-copy kernel), a random field, 6 steps: bitwise."""
    n, b, steps = 512, 16, 6
    h = 1.0 / n
    grid = L.CartesianGrid([n] * 3, [b] * 3, [0.0] * 3, [h] * 3).with_periodic([True] * 3)
    sim = L.Simulation(grid, L.FiniteDifference(), L.Heat(1.0), L.ForwardEuler(), sched, L.CudaAllocator("f64"))
    og = orc.Grid([n] * 3, [b] * 3, [0.0] * 3, [h] * 3, [True] * 3)
    os_ = orc.State(og, [1])
    u0 = np.random.default_rng(5).standard_normal((og.num_blocks(),) + og.slab_shape(1))
    sim.state.upload("u", u0)
    os_.set(0, u0)
    del u0
    dt = 0.15 * h * h
    sim.run(dt, steps, graph=True)
    t = os_.heat_run(0, 1.0, 0.0, dt, steps, THREADS)
    assert np.array_equal(sim.state.interior("u"), os_.interior(0))
    assert sim.time() == t
    del sim, os_
