"""Observation on the host: cell centres and the Parquet snapshot files.

The round-trip test restates the reference's tests/parquet.rs:91-139 (a 4x4
grid of 2x2 blocks, spacing 0.5, phi = 100 x + y, a static theta0 =
-(1000 y + x), cadence 2): per-epoch static file with x, y, level, patch and
theta0; snapshot files with step, t, epoch and phi in writer row order;
doubles bit for bit.  No device is used: the state is a host stand-in with
the device state's ``interior`` view.
"""
from fractions import Fraction

import numpy as np
import pyarrow.parquet as pq
import pytest

import legendre_b200 as L
from legendre_b200 import observe as O


def exact_center(g, i, h, o):
    # (g + i + 0.5) * h + o rounded once: the reference's mul_add
    return float(Fraction(float(g + i) + 0.5) * Fraction(h) + Fraction(o))


@pytest.mark.parametrize("cells,block,origin,spacing", [
    ((12,), (4,), (0.1,), (0.37,)),
    ((6, 9), (3, 3), (-1.3, 0.7), (0.4, 0.3)),
    ((4, 6, 4), (2, 3, 2), (0.01, -2.0, 5.5), (0.1, 1.0 / 3.0, 0.7)),
])
def test_cell_centers_are_the_references_fma(cells, block, origin, spacing):
    grid = L.CartesianGrid(list(cells), list(block), list(origin), list(spacing))
    got = O.cell_centers(grid)
    D = len(cells)
    nb = [c // b for c, b in zip(cells, block)]
    row = 0
    for b in range(int(np.prod(nb))):
        bc = [(b // int(np.prod(nb[:d]))) % nb[d] for d in range(D)]
        for idx in np.ndindex(*reversed(block)):
            idx = tuple(reversed(idx))  # dimension 0 fastest
            for d in range(D):
                assert got[d, row] == exact_center(bc[d] * block[d], idx[d], spacing[d], origin[d])
            row += 1


class HostState:
    """Host stand-in for a device state: named fields as (num_blocks, ny, nx) interiors."""

    def __init__(self, fields):
        self.fields = fields

    def interior(self, f):
        return self.fields[f]


def reference_state(grid):
    xy = O.cell_centers(grid)
    nb = grid.num_blocks()
    shape = (nb,) + tuple(reversed(grid.block_cells))
    phi = (100.0 * xy[0] + xy[1]).reshape(shape)  # exact: quarter multiples
    theta = -(1000.0 * xy[1] + xy[0]).reshape(shape)
    return HostState({"phi": phi, "theta0": theta}), xy


def test_snapshot_roundtrips_exactly(tmp_path):
    grid = L.CartesianGrid([4, 4], [2, 2], [0.0, 0.0], [0.5, 0.5])
    state, xy = reference_state(grid)
    obs = L.ParquetObserver(grid, [("phi", "phi")], 2, tmp_path).with_static([("theta0", "theta0")])
    # cadence: step 1 always fires, step 3 is skipped, step 4 fires
    obs.observe(1, 0.25, 0, grid, state)
    obs.observe(3, 0.75, 0, grid, state)
    obs.observe(4, 1.0, 0, grid, state)
    static = tmp_path / "static_0000000.parquet"
    snap1, snap3, snap4 = (tmp_path / f"snap_{s:07d}.parquet" for s in (1, 3, 4))
    assert static.exists() and snap1.exists() and snap4.exists()
    assert not snap3.exists()
    st = pq.read_table(static)
    assert st.column_names == ["x", "y", "level", "patch", "theta0"]
    assert np.array_equal(st["x"].to_numpy(), xy[0])
    assert np.array_equal(st["y"].to_numpy(), xy[1])
    assert np.array_equal(st["theta0"].to_numpy(), -(1000.0 * xy[1] + xy[0]))
    assert np.array_equal(st["level"].to_numpy(), np.zeros(16))
    assert np.array_equal(st["patch"].to_numpy(), np.repeat(np.arange(4.0), 4))
    for path, step, t in ((snap1, 1, 0.25), (snap4, 4, 1.0)):
        s = pq.read_table(path)
        assert s.column_names == ["step", "t", "epoch", "phi"]
        assert np.array_equal(s["phi"].to_numpy(), 100.0 * xy[0] + xy[1])
        assert np.array_equal(s["step"].to_numpy(), np.full(16, step, dtype=np.int64))
        assert np.array_equal(s["epoch"].to_numpy(), np.zeros(16, dtype=np.int64))
        assert np.array_equal(s["t"].to_numpy(), np.full(16, t))
        # required columns, SNAPPY
        assert all(not f.nullable for f in s.schema)
        md = pq.ParquetFile(path).metadata
        assert md.row_group(0).column(0).compression == "SNAPPY"
    # the row order is block-major: the first block's four cells come first
    assert list(xy[0][:4]) == [0.25, 0.75, 0.25, 0.75] and list(xy[1][:4]) == [0.25, 0.25, 0.75, 0.75]


def test_epoch_change_writes_a_new_static_file(tmp_path):
    grid = L.CartesianGrid([4, 4], [2, 2], [0.0, 0.0], [0.5, 0.5])
    state, _ = reference_state(grid)
    obs = L.ParquetObserver(grid, [("phi", "phi")], 2, tmp_path)
    obs.observe(1, 0.1, 0, grid, state)
    obs.observe(3, 0.3, 1, grid, state)  # off cadence: the epoch is noted
    obs.observe(4, 0.4, 1, grid, state)
    assert (tmp_path / "static_0000000.parquet").exists() and (tmp_path / "static_0000001.parquet").exists()
    assert np.array_equal(pq.read_table(tmp_path / "snap_0000004.parquet")["epoch"].to_numpy(), np.ones(16, np.int64))


def test_row_groups_hold_whole_blocks(tmp_path, monkeypatch):
    # groups flush once the bound is reached, at a block boundary
    monkeypatch.setattr(O, "ROWS_PER_GROUP", 10)
    grid = L.CartesianGrid([8, 6], [4, 3], [0.0, 0.0], [1.0, 1.0])  # 4 blocks of 12 cells
    xy = O.cell_centers(grid)
    sink = L.ParquetObserver(grid, [("phi", "phi")], 1, tmp_path)
    sink.consume(L.Snapshot(7, 0.5, 0, grid, {"phi": xy[0] * 3.0}))
    md = pq.ParquetFile(tmp_path / "snap_0000007.parquet").metadata
    assert [md.row_group(i).num_rows for i in range(md.num_row_groups)] == [12, 12, 12, 12]
    assert np.array_equal(pq.read_table(tmp_path / "snap_0000007.parquet")["phi"].to_numpy(), xy[0] * 3.0)


def test_runs_are_cut_at_the_observed_steps():
    from legendre_b200.core import observed_stretches

    # from step 0: step 1 fires, then every 5
    assert observed_stretches(0, 23, [5]) == [1, 4, 5, 5, 5, 3]
    # two cadences: the union of their steps
    assert observed_stretches(0, 12, [4, 6]) == [1, 3, 2, 2, 4]
    # resuming mid-run: no step 1, the next multiple first
    assert observed_stretches(7, 10, [5]) == [3, 5, 2]
    assert sum(observed_stretches(3, 100, [7, 11])) == 100


def test_async_observer_cadence_of_the_reference():
    # tests/model_c.rs:144-178: every 20 over 100 steps observes steps 1, 20,
    # 40, 60, 80 and 100 (delivery and the drain at shutdown run on the
    # device in tests/test_gpu_observe.py)
    from itertools import accumulate

    from legendre_b200.core import observed_stretches

    ends = list(accumulate(observed_stretches(0, 100, [20])))
    assert [s for s in ends if s == 1 or s % 20 == 0] == [1, 20, 40, 60, 80, 100]
    assert ends[-1] == 100


def test_runs_end_exactly_at_the_observed_steps_property():
    # every step an observer fires on ends a run, and no other step does
    # (except the last step of the call)
    from hypothesis import given, settings
    from hypothesis import strategies as st

    from legendre_b200.core import observed_stretches
    from legendre_b200.observe import fires

    @settings(max_examples=200, deadline=None)
    @given(st.integers(0, 60), st.integers(1, 80), st.lists(st.integers(1, 13), min_size=1, max_size=3))
    def check(k, n, everys):
        runs = observed_stretches(k, n, everys)
        assert all(r > 0 for r in runs) and sum(runs) == n
        ends, e = [], k
        for r in runs:
            e += r
            ends.append(e)
        fired = [s for s in range(k + 1, k + n + 1) if any(fires(s, c) for c in everys)]
        assert [s for s in ends if s in fired] == fired
        assert all(s in fired for s in ends[:-1])

    check()
