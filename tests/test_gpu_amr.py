"""AMR on the device against the AMR oracle (needs a GPU).

Bitwise for FP64 without noise: the patch hierarchy (regrids included), the
ghost fill, restriction, tagging and subcycled steps.  With noise, the
integer keys are exact and the states agree to 1e-12.
"""
import math

import numpy as np
import pytest

import legendre_b200 as L

pytestmark = pytest.mark.gpu


def make_pair(sched, orc, cells, block, h, ratios, patches=(), model="heat", integrator="subcycling", seed=0,
              noise=0.0, policy=None, kappa=0.7):
    base = L.CartesianGrid(cells, block, [0.0, 0.0], [h, h])
    grid = L.AmrGrid.from_patches(base, ratios, [[L.CellBox(lo, hi) for lv, lo, hi in patches if lv == l + 1]
                                                 for l in range(max([p[0] for p in patches], default=0))])
    if model == "heat":
        m, disc, params = L.Heat(kappa), L.FiniteDifference(), None
    else:
        m, disc, params = L.ModelC(0.06, 3.19, noise), L.FiniteVolume(), orc.modelc_params(noise=noise)
    integ = L.Subcycling(seed) if integrator == "subcycling" else L.EulerMaruyama(seed)
    adapt = None
    if policy is not None:
        adapt = L.BergerOliger(L.GradientTagger(m.__class__ is L.Heat and "u" or "phi", policy["threshold"]),
                               L.RegridPolicy(policy["every"], policy["buffer"],
                                              L.ClusterParams(policy["efficiency"], policy["min_width"])))
    dev = L.AmrSimulation(grid, disc, m, integ, sched, L.CudaAllocator("f64"), adapt)
    ref = orc.AmrSim(cells, block, h, ratios, patches, model=model, params=params, kappa=kappa,
                     integrator=integrator, seed=seed, wiener=noise != 0.0,
                     policy=None if policy is None else dict(policy, field=0))
    return dev, ref


def set_both(dev, ref, f, fn):
    slabs = ref.get(f)
    for b in range(ref.num_blocks):
        xs, ys = ref.centers(b)
        slabs[b][1:-1, 1:-1] = fn(xs, ys)
    ref.set(f, slabs)
    dev.set(f, slabs)


def same_state(dev, ref, nfields, interior=True, exact=True):
    assert dev.patches() == ref.patches()
    for f in range(nfields):
        for a, b in zip(dev.get(f), ref.get(f)):
            if interior:
                a, b = a[1:-1, 1:-1], b[1:-1, 1:-1]
            if exact:
                assert np.array_equal(a, b)
            else:
                assert np.allclose(a, b, rtol=1e-12, atol=1e-12)


def test_linear_field_ghosts_and_restriction(sched, orc):
    # tests/amr.rs:224-296 on the device, full slabs against the oracle
    dev, ref = make_pair(sched, orc, [8, 8], [4, 4], 0.5, [2], [(1, (4, 4), (8, 12)), (1, (8, 4), (12, 12))])
    set_both(dev, ref, 0, lambda x, y: (3.0 * x + 2.0) - y)
    for s in (dev, ref):
        slabs = s.get(0)
        slabs[0][3:5, 3:5] = 99.0
        s.set(0, slabs)
    dev.restrict(0)
    dev.fill_ghosts()
    ref.restrict(0)
    ref.fill_ghosts(0)
    same_state(dev, ref, 1, interior=False)


def test_tag_level_matches_oracle(sched, orc):
    dev, ref = make_pair(sched, orc, [32, 32], [16, 16], 0.5, [2], [(1, (16, 16), (40, 40))])
    gauss = lambda x, y: np.exp(-((x - 8.0) ** 2 + (y - 8.0) ** 2) / 3.0)
    set_both(dev, ref, 0, gauss)
    dev.fill_ghosts()
    ref.fill_ghosts(0)
    for level in (0, 1):
        assert dev.tag_level(0, level, 0.03) == sorted(ref.tag(0, 0.03, level))


TILED = [(1, (0, 0), (8, 16)), (1, (8, 0), (16, 16))]
INIT = staticmethod(lambda x, y: np.vectorize(math.cos)(0.6 * x) + np.vectorize(math.sin)(1.1 * y))


MODES = {"launches": {}, "graph": {"graph": True}, "persistent": {"persistent": True}}


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("integrator", ["subcycling", "global"])
def test_tiled_heat_bit_identical(sched, orc, integrator, mode):
    # tests/amr.rs:346-448 and 1016-1113 on the device
    dev, ref = make_pair(sched, orc, [8, 8], [8, 8], 0.5, [2], TILED, integrator=integrator)
    set_both(dev, ref, 0, lambda x, y: np.vectorize(math.cos)(0.6 * x) + np.vectorize(math.sin)(1.1 * y))
    dt = ref.suggested_dt()
    assert dev.stable_dt() == dt
    dev.run(dt, 25, **MODES[mode])
    ref.step(dt, 25)
    same_state(dev, ref, 1)
    assert dev.time() == ref.step(dt, 0)


HEAT_POLICY = dict(every=2, buffer=2, efficiency=0.7, min_width=4, threshold=0.03)


@pytest.mark.parametrize("mode", sorted(MODES))
def test_adaptive_subcycled_heat_bit_identical(sched, orc, mode):
    # tests/amr.rs:1115-1180 setup: regrids every 2 steps
    dev, ref = make_pair(sched, orc, [32, 32], [16, 16], 0.5, [2], [], policy=HEAT_POLICY)
    set_both(dev, ref, 0, lambda x, y: np.exp(-((x - 8.0) * (x - 8.0) + (y - 8.0) * (y - 8.0)) / 3.0))
    dt = ref.suggested_dt()
    dev.run(dt, 30, **MODES[mode])
    ref.step(dt, 30)
    assert dev.num_levels == 2 and dev.epoch == ref.epoch
    same_state(dev, ref, 1)


MC_POLICY = dict(every=4, buffer=2, efficiency=0.8, min_width=4, threshold=0.15)


def _seed(x, y):
    r = np.vectorize(math.hypot)(x - 0.4, y - 0.4)
    return np.maximum(-1.0, -np.vectorize(math.tanh)((r - 4.0) / math.sqrt(2.0)))


@pytest.mark.parametrize("mode", ["graph", "persistent"])
@pytest.mark.parametrize("integrator,steps", [("subcycling", 40), ("global", 60), ("subcycling", 41)])
def test_adaptive_model_c_bit_identical(sched, orc, integrator, steps, mode):
    # tests/amr.rs:918-989 and 1182-1228 setups
    dev, ref = make_pair(sched, orc, [48, 48], [24, 24], 0.4, [2], [], model="modelc", integrator=integrator,
                         seed=7, policy=MC_POLICY)
    set_both(dev, ref, 0, _seed)
    set_both(dev, ref, 1, lambda x, y: np.full_like(x, -0.7))
    dt = ref.suggested_dt()
    dev.run(dt, steps, **MODES[mode])
    ref.step(dt, steps)
    assert dev.num_levels == 2
    same_state(dev, ref, 2)


@pytest.mark.parametrize("mode", ["graph", "persistent"])
def test_adaptive_model_c_three_levels_with_noise(sched, orc, mode):
    dev, ref = make_pair(sched, orc, [64, 64], [32, 32], 0.4, [2, 2], [], model="modelc", seed=3, noise=0.02,
                         policy=dict(every=5, buffer=2, efficiency=0.8, min_width=4, threshold=0.1))
    set_both(dev, ref, 0, lambda x, y: np.maximum(-1.0, -np.vectorize(math.tanh)(
        (np.vectorize(math.hypot)(x - 12.8, y - 12.8) - 5.0) / math.sqrt(2.0))))
    set_both(dev, ref, 1, lambda x, y: np.full_like(x, -0.6))
    dt = ref.suggested_dt()
    dev.run(dt, 12, **MODES[mode])
    ref.step(dt, 12)
    assert dev.num_levels == ref.num_levels == 3
    same_state(dev, ref, 2, exact=False)


def test_persistent_barrier_timeout_returns_an_error_and_the_context_stays_usable(sched, orc):
    """The one bounded device wait: a grid barrier of the persistent launch
    told to give up at its first poll returns LG_ERR_TIMEOUT (no fault, no
    hang), and a fresh simulation on the same context then steps to the
    oracle's bits."""
    dev, ref0 = make_pair(sched, orc, [48, 48], [24, 24], 0.4, [2], [], model="modelc", integrator="subcycling",
                          seed=7, policy=MC_POLICY)
    set_both(dev, ref0, 0, _seed)
    set_both(dev, ref0, 1, lambda x, y: np.full_like(x, -0.7))
    dt = dev.stable_dt()
    dev.set_barrier_spin_limit(0)
    with pytest.raises(L.LegendreError) as err:
        dev.run(dt, 4, persistent=True)
    assert err.value.status == L._native.LG_ERR_TIMEOUT
    dev2, ref = make_pair(sched, orc, [48, 48], [24, 24], 0.4, [2], [], model="modelc", integrator="subcycling",
                          seed=7, policy=MC_POLICY)
    set_both(dev2, ref, 0, _seed)
    set_both(dev2, ref, 1, lambda x, y: np.full_like(x, -0.7))
    dev2.run(dt, 12, persistent=True)
    ref.step(dt, 12)
    same_state(dev2, ref, 2)
