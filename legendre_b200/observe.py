"""Observation of a running simulation: snapshots and Parquet output.

Mirrors the reference's two layers (src/core/observer.rs) and its Parquet
writer (src/io/parquet.rs):

* An *observer* has ``observe(step, t, epoch, grid, state)``, called by
  :class:`~legendre_b200.core.Simulation` after the steps it fires on
  (step 1 and every ``every`` steps, ``observer.rs:149-151``).
* A *snapshot sink* has ``consume(snapshot)`` and ``finish()`` and may do
  slow work (file IO, statistics).
* :class:`AsyncObserver` is the device form of the reference's
  ``AsyncObserver``: a ring of snapshot slots on the GPU and in pinned host
  memory (``lg_snapshot_ring_*``).  A capture is one gather kernel on the
  simulation's stream plus a copy on a stream of the ring's own; a background
  thread hands finished snapshots to the sinks and frees their slots.  The
  stepping stream never waits for the host: with every slot in flight the
  snapshot is dropped and counted (``observer.rs:17-25``).
* :class:`ParquetObserver` writes the reference's files: one
  ``static_{epoch:07}.parquet`` per grid epoch (x, y[, z], level, patch and
  any static fields) and one ``snap_{step:07}.parquet`` per snapshot (step,
  t, epoch and the dynamic fields), rows in block order with each block's
  interior cells dimension-0-fastest, SNAPPY, row groups of whole blocks
  flushed once 2^22 rows are gathered (``parquet.rs:150-215``).  It is an
  observer (synchronous) and a sink (behind an :class:`AsyncObserver`).
  Observing an ``AmrSimulation`` it writes every level's blocks, with their
  level and patch per cell, and a new static file at each regrid epoch
  (the reference's grid-aware path).
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N

ROWS_PER_GROUP = 1 << 22  # parquet.rs:60


def fires(step: int, every: int) -> bool:
    """The reference's snapshot cadence: step 1, then every ``every`` steps."""
    return step == 1 or (every > 0 and step % every == 0)


@dataclass
class Snapshot:
    """One observation: ``columns`` maps a field name to its values, one per
    interior cell in the Parquet row order (FP64).  Behind an
    :class:`AsyncObserver` the arrays are views of a pinned ring slot that is
    reused once ``consume`` returns: a sink that keeps data copies it."""

    step: int
    t: float
    epoch: int
    grid: object
    columns: Dict[str, np.ndarray]


def cell_centers(grid) -> np.ndarray:
    """(D, rows) cell centres of a Cartesian grid in the Parquet row order,
    computed by the library as the reference's ``cell_center`` does (one
    fused multiply-add per coordinate, cartesian.rs:589-597)."""
    D = len(grid.cells)
    rows = int(np.prod(grid.cells))
    out = np.empty((D, rows), dtype=np.float64)
    arr = lambda t, v: (t * D)(*v)
    N.check(N.lib.lg_cell_centers(D, arr(C.c_int64, grid.cells), arr(C.c_int64, grid.block_cells),
                                  arr(C.c_double, grid.origin), arr(C.c_double, grid.spacing),
                                  out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


def is_amr(sim) -> bool:
    """True for an AmrSimulation (blocks of several levels, regrid epochs)."""
    return hasattr(sim, "patches") and hasattr(sim, "centers")


def amr_columns(sim, names: Sequence[Tuple[str, object]]) -> Dict[str, np.ndarray]:
    """Columns of an AMR hierarchy in the writer's row order: blocks in
    order (level 0's, then each finer level's patches), each block's interior
    cells dimension-0-fastest."""
    out = {}
    for name, f in names:
        out[name] = np.concatenate([slab[1:-1, 1:-1].reshape(-1) for slab in sim.get(f)])
    return out


def amr_statics(sim):
    """x, y, level and patch of every cell of an AMR hierarchy, row order as
    amr_columns; x, y are the reference's cell centres (amr/grid.rs:389-395)."""
    xs, ys, lv, pt = [], [], [], []
    for b, (level, lo, hi) in enumerate(sim.patches()):
        x, y = sim.centers(b)
        xs.append(x.reshape(-1))
        ys.append(y.reshape(-1))
        lv.append(np.full(x.size, float(level)))
        pt.append(np.full(x.size, float(b)))
    return np.concatenate(xs), np.concatenate(ys), np.concatenate(lv), np.concatenate(pt)


def state_columns(state, names: Sequence[Tuple[str, object]]) -> Dict[str, np.ndarray]:
    """Columns of a device state read synchronously (download, then the
    interior of each block in row order)."""
    return {name: np.ascontiguousarray(state.interior(f), dtype=np.float64).reshape(-1) for name, f in names}


class ParquetObserver:
    """Snapshots of the dynamic ``fields`` -- a list of (column name, state
    field) -- every ``every`` steps plus step 1, into ``directory``."""

    def __init__(self, grid, fields: Sequence[Tuple[str, object]], every: int, directory):
        cells = grid.cells if hasattr(grid, "cells") else grid.base.cells
        if not 1 <= len(cells) <= 3:
            raise ValueError("the Parquet observer covers 1-, 2- and 3-D grids")
        if not fields:
            raise ValueError("no fields to observe")
        self.grid = grid
        self.dynamic = list(fields)
        self.statics: List[Tuple[str, object]] = []
        self.every = int(every)
        self.dir = os.fspath(directory)
        os.makedirs(self.dir, exist_ok=True)
        self.epoch = 0
        self.static_written = False

    def with_static(self, fields: Sequence[Tuple[str, object]]) -> "ParquetObserver":
        """Time-invariant fields written once per grid epoch (parquet.rs:112-116)."""
        self.statics = list(fields)
        return self

    def field_names(self) -> List[Tuple[str, object]]:
        """Every (column, field) the files need: the dynamic and static fields."""
        return self.dynamic + self.statics

    # ------------------------------------------------------------- writing
    @staticmethod
    def _groups(block_rows: Sequence[int]) -> List[Tuple[int, int]]:
        """Row groups as (start, rows): whole blocks, a group flushed once it
        holds ROWS_PER_GROUP rows or more (parquet.rs:150-215)."""
        out, start, n = [], 0, 0
        for r in block_rows:
            n += int(r)
            if n >= ROWS_PER_GROUP:
                out.append((start, n))
                start, n = start + n, 0
        if n:
            out.append((start, n))
        return out

    def _block_rows(self, amr=None) -> List[int]:
        if amr is not None:
            return [(hi[0] - lo[0]) * (hi[1] - lo[1]) for _, lo, hi in amr.patches()]
        bcells = int(np.prod(self.grid.block_cells))
        return [bcells] * (int(np.prod(self.grid.cells)) // bcells)

    def _write(self, path: str, cols: List[Tuple[str, object, np.ndarray]], block_rows: Sequence[int]):
        import pyarrow as pa
        import pyarrow.parquet as pq

        pa_type = {np.dtype(np.float64): pa.float64(), np.dtype(np.int64): pa.int64()}
        schema = pa.schema([pa.field(n, pa_type[np.dtype(dt)], nullable=False) for n, dt, _ in cols])
        with pq.ParquetWriter(path, schema, compression="snappy") as w:
            for lo, n in self._groups(block_rows):
                arrays = []
                for _, dt, v in cols:
                    a = np.full(n, v, dtype=dt) if np.isscalar(v) else v[lo:lo + n]
                    arrays.append(pa.array(a, type=pa_type[np.dtype(dt)]))
                w.write_table(pa.Table.from_arrays(arrays, schema=schema), row_group_size=n)

    def _write_static(self, columns: Dict[str, np.ndarray], amr=None):
        if amr is not None:  # the hierarchy's blocks: per-cell level and patch (parquet.rs:186-196)
            x, y, lv, pt = amr_statics(amr)
            cols = [("x", np.float64, x), ("y", np.float64, y), ("level", np.float64, lv), ("patch", np.float64, pt)]
        else:
            D = len(self.grid.cells)
            xyz = cell_centers(self.grid)
            bcells = int(np.prod(self.grid.block_cells))
            nb = int(np.prod(self.grid.cells)) // bcells
            cols = [(("x", "y", "z")[d], np.float64, xyz[d]) for d in range(D)]
            cols.append(("level", np.float64, np.zeros(nb * bcells)))
            cols.append(("patch", np.float64, np.repeat(np.arange(nb, dtype=np.float64), bcells)))
        cols += [(name, np.float64, columns[name]) for name, _ in self.statics]
        self._write(os.path.join(self.dir, f"static_{self.epoch:07d}.parquet"), cols, self._block_rows(amr))

    def write_snapshot(self, snap: Snapshot, amr=None) -> None:
        if snap.epoch != self.epoch:
            self.epoch = snap.epoch
            self.static_written = False
        if not self.static_written:
            self._write_static(snap.columns, amr)
            self.static_written = True
        cols = [("step", np.int64, np.int64(snap.step)), ("t", np.float64, np.float64(snap.t)),
                ("epoch", np.int64, np.int64(snap.epoch))]
        cols += [(name, np.float64, snap.columns[name]) for name, _ in self.dynamic]
        self._write(os.path.join(self.dir, f"snap_{snap.step:07d}.parquet"), cols, self._block_rows(amr))

    # ------------------------------------------------------ as an observer
    def observe(self, step: int, t: float, epoch: int, grid, state) -> None:
        if not fires(step, self.every):
            if epoch != self.epoch:
                self.epoch = epoch
                self.static_written = False
            return
        if epoch != self.epoch:
            self.grid = grid
        if is_amr(state):  # an AmrSimulation observes itself: blocks of every level
            cols = amr_columns(state, self.field_names())
            self.write_snapshot(Snapshot(step, t, epoch, grid, cols), amr=state)
            return
        cols = state_columns(state, self.field_names())
        self.write_snapshot(Snapshot(step, t, epoch, grid, cols))

    # ---------------------------------------------------------- as a sink
    def consume(self, snap: Snapshot) -> None:
        """Every snapshot handed over is written; the cadence belongs to the
        :class:`AsyncObserver` feeding it (construct with ``every = 1``)."""
        self.write_snapshot(snap)

    def finish(self) -> None:
        pass


class AsyncObserver:
    """Snapshots every ``every`` steps (and step 1) of ``fields`` -- a list of
    (column name, state field) -- moved off the device through a ring of
    ``nslots`` slots and handed to ``sinks`` on a background thread.

    The ring is bound to the first state observed; the state must outlive
    the observer.  ``close()`` drains the snapshots in flight, calls every
    sink's ``finish`` and frees the ring."""

    def __init__(self, every: int, nslots: int, sinks: Sequence, fields: Sequence[Tuple[str, object]]):
        if nslots < 1:
            raise ValueError("the ring needs at least one slot")
        self.every = int(every)
        self.nslots = int(nslots)
        self.sinks = list(sinks)
        self.fields = list(fields)
        self.handle = None
        self._state = None
        self._grid = None
        self._ctx = None
        self._closing = threading.Event()
        self._worker: Optional[threading.Thread] = None
        self._consumed = 0
        self._error: Optional[BaseException] = None

    # ----------------------------------------------------------- the ring
    def _bind(self, grid, state) -> None:
        idx = [state._index(f) for _, f in self.fields]
        arr = (C.c_int * len(idx))(*idx)
        h = C.c_void_p()
        N.check(N.lib.lg_snapshot_ring_create(state.handle, arr, len(idx), self.nslots, C.byref(h)),
                state.scheduler.handle)
        self.handle, self._state, self._grid, self._ctx = h, state, grid, state.scheduler.handle
        self._worker = threading.Thread(target=self._run, name="legendre-observer", daemon=True)
        self._worker.start()

    def stats(self) -> Tuple[int, int]:
        """(snapshots captured, snapshots dropped)."""
        if self.handle is None:
            return 0, 0
        cap, drop, rows = C.c_int64(), C.c_int64(), C.c_int64()
        N.check(N.lib.lg_snapshot_ring_stats(self.handle, C.byref(cap), C.byref(drop), C.byref(rows)), self._ctx)
        return cap.value, drop.value

    @property
    def dropped_snapshots(self) -> int:
        """Snapshots skipped because every slot was still in flight."""
        return self.stats()[1]

    # ------------------------------------------------------- observer side
    def observe(self, step: int, t: float, epoch: int, grid, state) -> None:
        if not fires(step, self.every):
            return
        if self.handle is None:
            self._bind(grid, state)
        elif state is not self._state:
            raise ValueError("an AsyncObserver serves the one state it was bound to")
        slot = C.c_int()
        N.check(N.lib.lg_snapshot_ring_capture(self.handle, int(step), float(t), int(epoch), C.byref(slot)),
                self._ctx)

    # ----------------------------------------------------------- consumer
    def _run(self) -> None:
        slot, step, t, epoch = C.c_int(), C.c_int64(), C.c_double(), C.c_int64()
        cols = C.POINTER(C.c_double)()
        nf = len(self.fields)
        while True:
            rc = N.lib.lg_snapshot_ring_poll(self.handle, 20, C.byref(slot), C.byref(step), C.byref(t),
                                             C.byref(epoch), C.byref(cols))
            if rc == N.LG_ERR_TIMEOUT:
                if self._closing.is_set() and self._consumed >= self.stats()[0]:
                    break
                continue
            if rc != N.LG_OK:
                self._error = N.LegendreError(rc, N.lib.lg_last_error(self._ctx).decode())
                break
            rows = self.stats_rows()
            block = np.ctypeslib.as_array(cols, shape=(nf * rows,)).reshape(nf, rows)
            snap = Snapshot(step.value, t.value, epoch.value, self._grid,
                            {name: block[k] for k, (name, _) in enumerate(self.fields)})
            try:
                for sink in self.sinks:
                    sink.consume(snap)
            except BaseException as e:  # a failing sink ends observation, not the run
                self._error = e
            finally:
                N.lib.lg_snapshot_ring_release(self.handle, slot.value)
                self._consumed += 1
            if self._error is not None:
                break

    def stats_rows(self) -> int:
        cap, drop, rows = C.c_int64(), C.c_int64(), C.c_int64()
        N.check(N.lib.lg_snapshot_ring_stats(self.handle, C.byref(cap), C.byref(drop), C.byref(rows)), self._ctx)
        return rows.value

    def close(self) -> None:
        """Drain the snapshots in flight, finish the sinks, free the ring;
        re-raises an error a sink or the ring reported."""
        if self.handle is not None:
            self._closing.set()
            self._worker.join()
            N.lib.lg_snapshot_ring_destroy(self.handle)
            self.handle = None
        for sink in self.sinks:
            sink.finish()
        self.sinks = []
        if self._error is not None:
            e, self._error = self._error, None
            raise e

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
