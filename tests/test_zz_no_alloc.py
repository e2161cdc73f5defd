"""The allocation-free tagging entry point (``lg_amr_tag_level_static``)
against ``lg_amr_tag_level``, through the C-ABI (needs a GPU).

Collected last: the entry point's scratch is a static device array shared
by the whole process, so it must give the same answer after every other
test has run as it does alone.
"""
import ctypes as C
import math

import numpy as np
import pytest

import legendre_b200 as L
from legendre_b200 import _native as N

pytestmark = pytest.mark.gpu

STATIC_CELLS = 1 << 18  # the scratch's stated capacity, in cells of one level


def _sim(sched, cells, block, patches):
    base = L.CartesianGrid([cells, cells], [block, block], [0.0, 0.0], [0.4, 0.4])
    grid = L.AmrGrid.from_patches(base, [2], [[L.CellBox(lo, hi) for lo, hi in patches]])
    model = L.ModelC(0.05, 3.19, 0.0)
    sim = L.AmrSimulation(grid, L.FiniteVolume(), model, L.Subcycling(0), sched, L.CudaAllocator("f64"))
    c = cells * 0.4 / 2.0
    phi = sim.get("phi")
    for k in range(sim.num_blocks):
        xs, ys = sim.centers(k)
        phi[k][1:-1, 1:-1] = np.maximum(-1.0, -np.tanh((np.hypot(xs - c, ys - c) - 4.0) / math.sqrt(2.0)))
    sim.set("phi", phi)
    sim.fill_ghosts()
    return sim


def _tag(fn, sim, level, threshold, cap):
    out = np.zeros(2 * max(cap, 1), dtype=np.int64)
    count = C.c_int64(-1)
    rc = fn(sim.handle, 0, level, threshold, out.ctypes.data_as(C.POINTER(C.c_int64)), cap, C.byref(count))
    return rc, count.value, out


def test_static_tagging_matches_the_allocating_entry_point(sched):
    sim = _sim(sched, 64, 32, [((40, 40), (88, 88))])
    cap = 1 << 16
    for level in (0, 1):
        for _ in range(2):  # two calls in a row: the scratch's counter restarts at zero
            rc_a, n_a, a = _tag(N.lib.lg_amr_tag_level, sim, level, 0.05, cap)
            rc_s, n_s, s = _tag(N.lib.lg_amr_tag_level_static, sim, level, 0.05, cap)
            assert rc_a == N.LG_OK and rc_s == N.LG_OK, N.lib.lg_last_error(sched.handle)
            assert n_s == n_a > 0
            assert np.array_equal(s[:2 * n_s], a[:2 * n_a])


def test_static_tagging_rejects_a_level_beyond_the_scratch(sched):
    sim = _sim(sched, 1024, 32, [((1000, 1000), (1048, 1048))])  # level 0: 1024^2 cells
    rc, _, _ = _tag(N.lib.lg_amr_tag_level_static, sim, 0, 0.05, 16)
    assert rc == N.LG_ERR_INVALID
    assert f"at most {STATIC_CELLS}" in N.lib.lg_last_error(sched.handle).decode()
    rc, n, _ = _tag(N.lib.lg_amr_tag_level_static, sim, 1, 0.05, 1 << 12)  # 48^2 cells at level 1: accepted
    assert rc == N.LG_OK and n >= 0


def test_static_tagging_reports_a_short_output_buffer(sched):
    sim = _sim(sched, 64, 32, [((40, 40), (88, 88))])
    rc_a, n_a, _ = _tag(N.lib.lg_amr_tag_level, sim, 0, 0.05, 1 << 16)
    assert rc_a == N.LG_OK and n_a > 1
    rc, n, _ = _tag(N.lib.lg_amr_tag_level_static, sim, 0, 0.05, n_a - 1)
    assert rc == N.LG_ERR_INVALID and n == n_a
    rc, n, _ = _tag(N.lib.lg_amr_tag_level_static, sim, 0, 0.05, n_a)
    assert rc == N.LG_OK and n == n_a
