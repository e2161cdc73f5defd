"""The AMR oracle against the reference's own AMR tests (CPU only).

Each test restates one of src/geometry/amr/cluster.rs:283-524 or
tests/amr.rs, citing it; together they pin the oracle's restatement of the
reference's adaptive path before it checks the CUDA library.
"""
import math

import numpy as np
import pytest


def art(rows):
    return [(c, r) for r, row in enumerate(rows) for c, ch in enumerate(row) if ch == "x"]


def cover_disjoint(flags, boxes):
    for f in flags:
        n = sum(all(lo[d] <= f[d] < hi[d] for d in range(len(f))) for lo, hi in boxes)
        assert n == 1, (f, boxes)
    for i, (alo, ahi) in enumerate(boxes):
        for blo, bhi in boxes[i + 1:]:
            assert not all(alo[d] < bhi[d] and blo[d] < ahi[d] for d in range(len(alo)))


def cells(boxes):
    return sum(int(np.prod([h - l for l, h in zip(lo, hi)])) for lo, hi in boxes)


def test_cluster_dense_rectangle(orc):
    # cluster.rs:320-331
    flags = art(["xxxx", "xxxx", "xxxx"])
    assert orc.cluster(flags, 0.8, 4) == [((0, 0), (4, 3))]


def test_cluster_islands_split_at_holes(orc):
    # cluster.rs:333-346
    flags = art(["xx....xxx", "xx....xxx", "......xxx"])
    boxes = orc.cluster(flags, 0.8, 4)
    assert len(boxes) == 2
    cover_disjoint(flags, boxes)
    assert cells(boxes) == len(flags)


def test_cluster_l_shape_splits_at_inflection(orc):
    # cluster.rs:348-374
    flags = art(["xx......"] * 4 + ["xxxxxxxx"] * 2)
    boxes = orc.cluster(flags, 0.95, 2)
    cover_disjoint(flags, boxes)
    assert cells(boxes) == len(flags) and len(boxes) == 2


def test_cluster_v_shape(orc):
    # cluster.rs:376-395
    flags = art(["x.....x", "x.....x", ".x...x.", ".x...x.", "..x.x..", "..xxx.."])
    boxes = orc.cluster(flags, 0.7, 1)
    cover_disjoint(flags, boxes)
    assert len(flags) / cells(boxes) >= 0.7


def test_cluster_diagonal_stripe(orc):
    # cluster.rs:397-431
    flags = [(i, i) for i in range(8)]
    boxes = orc.cluster(flags, 0.8, 1)
    cover_disjoint(flags, boxes)
    assert len(flags) / cells(boxes) >= 0.8
    boxes = orc.cluster(flags, 0.8, 2)
    cover_disjoint(flags, boxes)
    for lo, hi in boxes:
        n = sum(all(lo[d] <= f[d] < hi[d] for d in range(2)) for f in flags)
        assert n / cells([(lo, hi)]) >= 0.5


def test_cluster_three_dimensional_islands(orc):
    # cluster.rs:437-455
    flags = [(x, y, z + dz) for x in range(2) for y in range(2) for z in range(2) for dz in (0, 6)]
    boxes = orc.cluster(flags, 0.8, 4)
    assert len(boxes) == 2 and cells(boxes) == 16
    cover_disjoint(flags, boxes)


def test_cluster_order_independent(orc):
    # cluster.rs:457-480 (shuffle by the counter-based mixer)
    flags = art(["xx....xxx", "xx..x.xxx", "....x.xxx"])
    b = list(flags)
    for i in range(len(b) - 1, 0, -1):
        j = orc.splitmix64(orc.mix_key(9, [i])) % (i + 1)
        b[i], b[j] = b[j], b[i]
    assert sorted(orc.cluster(flags, 0.8, 1)) == sorted(orc.cluster(b, 0.8, 1))


def test_cluster_empty(orc):
    assert orc.cluster([], 0.8, 4) == []


def test_from_patches_errors(orc):
    # amr/grid.rs:90-196 error paths
    with pytest.raises(ValueError):  # overlap
        orc.AmrSim([8, 8], [8, 8], 0.5, [2], [(1, (4, 4), (8, 8)), (1, (6, 6), (10, 10))])
    with pytest.raises(ValueError):  # misaligned
        orc.AmrSim([8, 8], [8, 8], 0.5, [2], [(1, (3, 4), (8, 8))])
    with pytest.raises(ValueError):  # not nested (outside the domain)
        orc.AmrSim([8, 8], [8, 8], 0.5, [2], [(1, (12, 12), (18, 18))])
    with pytest.raises(ValueError):  # more levels than ratios
        orc.AmrSim([8, 8], [8, 8], 0.5, [2], [(2, (4, 4), (8, 8))])


def _fill_by_center(sim, f, fn):
    slabs = sim.get(f)
    for b in range(sim.num_blocks):
        xs, ys = sim.centers(b)
        slabs[b][1:-1, 1:-1] = fn(xs, ys)
    sim.set(f, slabs)


def test_linear_field_ghosts_and_restriction_are_exact(orc):
    # tests/amr.rs:224-296
    lin = lambda x, y: (3.0 * x + 2.0) - y  # 3.0.mul_add(x, 2.0) - y up to rounding (tolerance 1e-12)
    sim = orc.AmrSim([8, 8], [4, 4], 0.5, [2], [(1, (4, 4), (8, 12)), (1, (8, 4), (12, 12))])
    _fill_by_center(sim, 0, lin)
    slabs = sim.get(0)
    slabs[0][1 + 2:1 + 4, 1 + 2:1 + 4] = 99.0  # corrupt coarse cells beneath the patches (block 0)
    sim.set(0, slabs)
    sim.restrict(0)
    sim.fill_ghosts(0)
    slabs = sim.get(0)
    for b in range(sim.num_blocks):
        lv, lo, hi = sim.patch(b)
        if lv != 1:
            continue
        nx, ny = hi[0] - lo[0], hi[1] - lo[1]
        for j in range(-1, ny + 1):
            for i in range(-1, nx + 1):
                if 0 <= i < nx and 0 <= j < ny:
                    continue
                x = (lo[0] + i + 0.5) * 0.25
                y = (lo[1] + j + 0.5) * 0.25
                assert abs(slabs[b][j + 1, i + 1] - lin(x, y)) <= 1e-12
    xs, ys = sim.centers(0)
    assert np.all(np.abs(slabs[0][1:-1, 1:-1] - lin(xs, ys)) <= 1e-12)


def _fine_field(sim, nfine):
    out = np.zeros((nfine, nfine))
    slabs = sim.get(0)
    for b in range(sim.num_blocks):
        lv, lo, hi = sim.patch(b)
        if lv == 1:
            out[lo[1]:hi[1], lo[0]:hi[0]] = slabs[b][1:-1, 1:-1]
    return out


def _uniform_heat(orc, init, kappa, hf, dt, steps):
    from util import centers, with_ghosts
    g = orc.Grid([16, 16], [8, 16], [0.0, 0.0], [hf, hf])
    st = orc.State(g, [1])
    x = centers([16, 16], [8, 16], [0.0, 0.0], [hf, hf], 0)
    y = centers([16, 16], [8, 16], [0.0, 0.0], [hf, hf], 1)
    st.set(0, with_ghosts(init(x, y), 1))
    st.heat_run(0, kappa, 0.0, dt, steps)
    u = st.interior(0)  # (2 blocks, 16, 8)
    return np.concatenate([u[0], u[1]], axis=1)


TILED = [(1, (0, 0), (8, 16)), (1, (8, 0), (16, 16))]


def test_full_fine_tiling_matches_uniform_grid_bitwise(orc):
    # tests/amr.rs:346-448 (global dt, forward Euler heat)
    kappa, hf = 0.7, 0.25
    dt = 0.2 * hf * hf / kappa
    init = lambda x, y: np.vectorize(math.cos)(0.7 * x) + np.vectorize(math.sin)(1.3 * y)
    sim = orc.AmrSim([8, 8], [8, 8], 0.5, [2], TILED, kappa=kappa, integrator="global")
    _fill_by_center(sim, 0, init)
    sim.step(dt, 100)
    assert np.array_equal(_fine_field(sim, 16), _uniform_heat(orc, init, kappa, hf, dt, 100))


def test_fully_tiled_subcycled_fine_matches_uniform_fine_bitwise(orc):
    # tests/amr.rs:1016-1113
    kappa = 0.7
    init = lambda x, y: np.vectorize(math.cos)(0.6 * x) + np.vectorize(math.sin)(1.1 * y)
    sim = orc.AmrSim([8, 8], [8, 8], 0.5, [2], TILED, kappa=kappa, integrator="subcycling")
    dt_coarse = sim.suggested_dt()
    _fill_by_center(sim, 0, init)
    sim.step(dt_coarse, 25)
    ref = _uniform_heat(orc, init, kappa, 0.25, dt_coarse / 4.0, 100)
    assert np.array_equal(_fine_field(sim, 16), ref)


def _adaptive_heat(orc, threads):
    # tests/amr.rs:1115-1180
    sim = orc.AmrSim([32, 32], [16, 16], 0.5, [2], [], kappa=0.7, integrator="subcycling",
                     policy=dict(every=2, buffer=2, efficiency=0.7, min_width=4, threshold=0.03, field=0))
    sim.threads(threads)
    def gauss(x, y):
        dx, dy = x - 8.0, y - 8.0
        return np.exp(-(dx * dx + dy * dy) / 3.0)
    _fill_by_center(sim, 0, gauss)
    sim.step(sim.suggested_dt(), 30)
    return np.concatenate([s[1:-1, 1:-1].ravel() for (b, s) in enumerate(sim.get(0)) if sim.patch(b)[0] == 0]), sim


def test_adaptive_subcycled_run_is_thread_independent(orc):
    a, sa = _adaptive_heat(orc, 1)
    b, _ = _adaptive_heat(orc, 4)
    assert np.array_equal(a, b)
    assert sa.num_levels == 2 and sa.epoch >= 1


def _model_c_adaptive(orc, integrator, steps):
    sim = orc.AmrSim([48, 48], [24, 24], 0.4, [2], [], model="modelc", params=orc.modelc_params(),
                     integrator=integrator, seed=7 if integrator == "global" else 0,
                     policy=dict(every=4, buffer=2, efficiency=0.8, min_width=4, threshold=0.15, field=0))
    # ModelC::initialize on the base grid (phasefield.rs:180-189): one seed at (0.4, 0.4), r = 4, u0 = 0.7
    phi = sim.get(0)
    u = sim.get(1)
    for b in range(sim.num_blocks):
        xs, ys = sim.centers(b)
        r = np.vectorize(math.hypot)(xs - 0.4, ys - 0.4)
        phi[b][1:-1, 1:-1] = np.maximum(-1.0, -np.vectorize(math.tanh)((r - 4.0) / math.sqrt(2.0)))
        u[b][1:-1, 1:-1] = -0.7
    sim.set(0, phi)
    sim.set(1, u)
    sim.step(sim.suggested_dt(), steps)
    return sim


def test_dendrite_interface_is_tracked_by_refinement(orc):
    # tests/amr.rs:918-989 (global-dt Euler-Maruyama)
    sim = _model_c_adaptive(orc, "global", 150)
    assert sim.num_levels == 2
    refined = sum((hi[0] - lo[0]) * (hi[1] - lo[1]) for lv, lo, hi in sim.patches() if lv == 1)
    assert 0 < refined < 96 * 96
    phi = sim.get(0)
    fine = {}
    for b, (lv, lo, hi) in enumerate(sim.patches()):
        assert np.all(np.isfinite(phi[b][1:-1, 1:-1])) and np.all(np.abs(phi[b][1:-1, 1:-1]) < 1.2)
    for b, (lv, lo, hi) in enumerate(sim.patches()):
        if lv != 0:
            continue
        v = phi[b]
        gx = 0.5 * (v[1:-1, 2:] - v[1:-1, :-2])
        gy = 0.5 * (v[2:, 1:-1] - v[:-2, 1:-1])
        for j, i in zip(*np.nonzero(np.maximum(np.abs(gx), np.abs(gy)) > 0.2)):
            cx, cy = (lo[0] + i) * 2, (lo[1] + j) * 2
            assert any(l2 == 1 and lo2[0] <= cx < hi2[0] and lo2[1] <= cy < hi2[1] for l2, lo2, hi2 in sim.patches())


def test_model_c_subcycled_dendrite_is_physical(orc):
    # tests/amr.rs:1182-1228
    sim = _model_c_adaptive(orc, "subcycling", 40)
    assert sim.num_levels == 2
    for s in sim.get(0):
        assert np.all(np.isfinite(s[1:-1, 1:-1])) and np.all(np.abs(s[1:-1, 1:-1]) < 1.2)
