"""The AMR oracle against the reference's adaptive-policy tests
(tests/amr.rs:487-905), on the CPU: a refined run stays physical, the first
step refines around the feature, the adaptive run beats the uniform-coarse
one against a restricted uniform-fine reference by the reference's own
published figures, and migration is exact on linear fields.  The device AMR
path is bit-identical to this oracle (tests/test_gpu_amr.py)."""
import math

import numpy as np
import pytest

from legendre_b200.rng import fma
from util import centers, with_ghosts

KAPPA = 0.7


def gaussian(x, y, w):
    dx, dy = x - 4.0, y - 4.0
    return math.exp(-fma(dx, dx, dy * dy) / w)


def fill_amr(sim, fn):
    slabs = sim.get(0)
    for b in range(sim.num_blocks):
        xs, ys = sim.centers(b)
        ny, nx = xs.shape
        for j in range(ny):
            for i in range(nx):
                slabs[b][1 + j, 1 + i] = fn(xs[j, i], ys[j, i])
    sim.set(0, slabs)


def interiors(sim, level=None):
    return [s[1:-1, 1:-1] for (lv, _, _), s in zip(sim.patches(), sim.get(0)) if level is None or lv == level]


# the reference's policy(): GradientTagger{"u", 0.05}, RegridPolicy{every 4,
# buffer 2, ClusterParams{0.7, 2}} (tests/amr.rs:563-577)
POLICY = dict(every=4, buffer=2, efficiency=0.7, min_width=2, threshold=0.05, field=0)


def test_interface_run_stays_physical(orc):
    # tests/amr.rs:487-543: one fine patch over a Gaussian bump, forward Euler
    dt = 0.2 * 0.25 * 0.25 / KAPPA
    sim = orc.AmrSim([16, 16], [8, 8], 0.5, [2], [(1, (8, 8), (24, 24))], kappa=KAPPA, integrator="global")
    fill_amr(sim, lambda x, y: gaussian(x, y, 1.5))
    sim.step(dt, 200)
    v = np.concatenate([s.ravel() for s in interiors(sim)])
    assert np.all(np.isfinite(v))
    assert v.max() < 0.9, "heat must decay from the initial peak of 1"
    assert v.max() > 0.0 and v.min() > -1e-9, "maximum principle"


def test_initial_regrid_refines_around_the_feature(orc):
    # tests/amr.rs:579-680
    dt = 0.2 * 0.25 * 0.25 / KAPPA
    sim = orc.AmrSim([16, 16], [8, 8], 0.5, [2], [], kappa=KAPPA, integrator="global", policy=POLICY)
    g = lambda x, y: gaussian(x, y, 0.4)
    fill_amr(sim, g)
    sim.step(dt)  # step 0 regrids from the initial conditions
    assert sim.num_levels == 2, "the bump must trigger refinement"
    boxes = [(lo, hi) for lv, lo, hi in sim.patches() if lv == 1]
    for cy in range(16):
        for cx in range(16):
            c0, c1 = fma(0.5, float(cx), 0.25), fma(0.5, float(cy), 0.25)
            gx = (g(c0 + 0.5, c1) - g(c0 - 0.5, c1)) / 2.0
            gy = (g(c0, c1 + 0.5) - g(c0, c1 - 0.5)) / 2.0
            if max(abs(gx), abs(gy)) > 0.06:
                fx, fy = 2 * cx, 2 * cy
                assert any(lo[0] <= fx < hi[0] and lo[1] <= fy < hi[1] for lo, hi in boxes), (cx, cy)
    sim.step(dt, 8)
    assert sim.num_levels == 2, "feature still present, still refined"
    v = np.concatenate([s.ravel() for s in interiors(sim)])
    assert np.all(np.isfinite(v)) and v.min() >= -1e-9 and v.max() <= 1.0


def uniform_heat(orc, n, block, h, dt, steps, fn):
    grid = orc.Grid([n, n], [block, block], [0.0, 0.0], [h, h])
    st = orc.State(grid, [1])
    x = centers([n, n], [block, block], [0.0, 0.0], [h, h], 0)
    y = centers([n, n], [block, block], [0.0, 0.0], [h, h], 1)
    st.set(0, with_ghosts(np.vectorize(fn)(x, y), 1))
    st.heat_run(0, KAPPA, 0.0, dt, steps)
    return st.interior(0), x, y


def test_adaptive_beats_coarse_against_fine_reference(orc):
    # tests/amr.rs:682-790, with the reference's published errors and
    # refined-cell count
    dt, steps = 0.2 * 0.25 * 0.25 / KAPPA, 60
    g = lambda x, y: gaussian(x, y, 0.4)
    fine, fx, fy = uniform_heat(orc, 32, 16, 0.25, dt, steps, g)
    reference = np.zeros((16, 16))
    for b in range(fine.shape[0]):
        for j in range(16):
            for i in range(16):
                cx, cy = int(fx[b, j, i] / 0.5), int(fy[b, j, i] / 0.5)
                reference[cy, cx] = fma(fine[b, j, i], 0.25, reference[cy, cx])
    coarse, _, _ = uniform_heat(orc, 16, 8, 0.5, dt, steps, g)

    sim = orc.AmrSim([16, 16], [8, 8], 0.5, [2], [], kappa=KAPPA, integrator="global", policy=POLICY)
    fill_amr(sim, g)
    refined = 0
    for _ in range(steps):
        sim.step(dt)
        refined = max(refined, sum((hi[0] - lo[0]) * (hi[1] - lo[1]) for lv, lo, hi in sim.patches() if lv == 1))
    sim.restrict(0)
    err_adaptive = err_coarse = 0.0
    for b, ((lv, lo, hi), s) in enumerate(zip(sim.patches(), sim.get(0))):
        if lv != 0:
            continue
        for j in range(hi[1] - lo[1]):
            for i in range(hi[0] - lo[0]):
                ref = reference[lo[1] + j, lo[0] + i]
                err_adaptive = max(err_adaptive, abs(s[1 + j, 1 + i] - ref))
                err_coarse = max(err_coarse, abs(coarse[b, j, i] - ref))
    assert err_adaptive == pytest.approx(0.001680900, abs=1e-6)
    assert err_coarse == pytest.approx(0.003716000, abs=1e-6)
    assert refined == 400, "refinement must stay partial"


def test_migration_preserves_linear_fields_exactly(orc):
    # tests/amr.rs:792-905: a forced refinement box [2,6)^2 (prolongation
    # path), then the box shifted to [4,8)^2 (copy of the overlap, prolongation
    # of the rest), buffer 0, ClusterParams{0.9, 2}; a linear field is kept
    # to 1e-12 (the reference's model is frozen; no step runs here)
    lin = lambda x, y: fma(3.0, x, 2.0) - y
    sim = orc.AmrSim([16, 16], [8, 8], 0.5, [2], [], kappa=KAPPA, integrator="global")
    fill_amr(sim, lin)
    box = lambda s: [(x, y) for y in range(2 + s, 6 + s) for x in range(2 + s, 6 + s)]
    assert sim.regrid_flags(box(0), 0, 0.9, 2)
    assert sim.regrid_flags(box(2), 0, 0.9, 2)
    assert sim.num_levels == 2
    fine = [b for b, (lv, _, _) in enumerate(sim.patches()) if lv == 1]
    assert fine
    slabs = sim.get(0)
    for b in fine:
        assert sim.patch(b)[1:] == ((8, 8), (16, 16)), "shifted box expected"
        xs, ys = sim.centers(b)
        for j in range(xs.shape[0]):
            for i in range(xs.shape[1]):
                want = lin(xs[j, i], ys[j, i])
                assert slabs[b][1 + j, 1 + i] == pytest.approx(want, rel=1e-12, abs=1e-12)
