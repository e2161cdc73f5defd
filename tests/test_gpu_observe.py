"""Snapshots through the device ring (AsyncObserver) on a GPU.

* Every snapshot equals the state of a twin run at its step, bit for bit
  (FP64, FP32 widened to FP64, 2-D Model C and 3-D heat), with step and time;
  the sinks see every snapshot and their finish() at shutdown
  (tests/model_c.rs:144-178).
* When the sink falls behind, snapshots are dropped and counted; the run
  itself is unchanged bit for bit, and the snapshots that did go through are
  the right ones.
* Parquet files written behind the ring equal those of the synchronous
  observer.
"""
import threading

import numpy as np
import pyarrow.parquet as pq
import pytest

import legendre_b200 as L
from util import with_ghosts

pytestmark = pytest.mark.gpu

H = 0.4


def modelc_sim(sched, dtype="f64", noise=0.02, cells=(64, 96), block=(32, 32), seed=3):
    grid = L.CartesianGrid(list(cells), list(block), [0.0, 0.0], [H, H])
    model = L.ModelC(0.05, 3.19, noise)
    model.d_thermal = 2.0
    sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(seed), sched, L.CudaAllocator(dtype))
    init = sim if dtype == "f64" else L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(seed), sched,
                                                   L.CudaAllocator("f64"))
    model.initialize_grains(grid, init.state, [L.Grain((cells[0] * H / 2, cells[1] * H / 2), 4.0)], 0.55)
    if init is not sim:  # FP32: a cast copy of the FP64 initial state
        for f in ("phi", "u"):
            sim.state.upload(f, init.state.download(f).astype(np.float32))
    return sim


def heat_sim(sched, cells=(12, 8, 16), block=(4, 4, 8)):
    grid = L.CartesianGrid(list(cells), list(block), [0.0] * 3, [0.1] * 3).with_periodic([True, False, True])
    sim = L.Simulation(grid, L.FiniteDifference(), L.Heat(0.7), L.ForwardEuler(), sched, L.CudaAllocator("f64"))
    rng = np.random.default_rng(5)
    sim.state.upload("u", with_ghosts(rng.standard_normal((grid.num_blocks(),) + tuple(reversed(block))), 1))
    return sim


class Collect:
    def __init__(self, gate=None):
        self.snaps, self.finished, self.gate = [], False, gate

    def consume(self, s):
        if self.gate is not None:
            self.gate.wait(30.0)
        self.snaps.append((s.step, s.t, s.epoch, {k: v.copy() for k, v in s.columns.items()}))

    def finish(self):
        self.finished = True


def twin_states(make, dt, steps, names):
    """{step: (t, {name: interior in row order})} of a run without observers."""
    sim = make()
    out = {}
    for k in range(1, steps + 1):
        sim.run(dt, 1)
        out[k] = (sim.time(), {n: sim.state.interior(f).astype(np.float64).reshape(-1) for n, f in names})
    return sim, out


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_snapshots_equal_the_state_at_their_steps(sched, dtype):
    names = [("phi", "phi"), ("u", "u")]
    make = lambda: modelc_sim(sched, dtype)
    dt = 0.01
    _, ref = twin_states(make, dt, 23, names)
    sim = make()
    sink = Collect()
    obs = L.AsyncObserver(every=5, nslots=8, sinks=[sink], fields=names)
    sim.add_observer(obs)
    sim.run(dt, 23, graph=True)
    obs.close()
    assert sink.finished
    assert [s[0] for s in sink.snaps] == [1, 5, 10, 15, 20]
    assert obs.dropped_snapshots == 0
    for step, t, epoch, cols in sink.snaps:
        assert t == ref[step][0] and epoch == 0
        for n, _ in names:
            assert np.array_equal(cols[n], ref[step][1][n]), (step, n)


def test_three_dimensional_snapshots(sched):
    names = [("u", "u")]
    make = lambda: heat_sim(sched)
    dt = 0.15 * 0.01 / 0.7
    _, ref = twin_states(make, dt, 9, names)
    sim = make()
    sink = Collect()
    obs = L.AsyncObserver(every=3, nslots=4, sinks=[sink], fields=names)
    sim.add_observer(obs)
    sim.run(dt, 9)
    obs.close()
    assert [s[0] for s in sink.snaps] == [1, 3, 6, 9]
    for step, t, _, cols in sink.snaps:
        assert np.array_equal(cols["u"], ref[step][1]["u"])


def test_a_slow_sink_drops_snapshots_not_steps(sched):
    names = [("phi", "phi")]
    make = lambda: modelc_sim(sched)
    dt = 0.01
    plain, ref = twin_states(make, dt, 40, names)
    sim = make()
    gate = threading.Event()
    sink = Collect(gate)
    obs = L.AsyncObserver(every=2, nslots=2, sinks=[sink], fields=names)
    sim.add_observer(obs)
    sim.run(dt, 40)
    sched.sync()
    gate.set()
    obs.close()
    captured, dropped = len(sink.snaps), None
    fired = [1] + list(range(2, 41, 2))
    assert captured >= 1 and captured < len(fired)
    dropped = len(fired) - captured
    steps = [s[0] for s in sink.snaps]
    assert steps == sorted(steps) and set(steps) <= set(fired)
    for step, t, _, cols in sink.snaps:
        assert np.array_equal(cols["phi"], ref[step][1]["phi"])
    assert dropped > 0
    for f in ("phi", "u"):
        assert np.array_equal(sim.state.download(f), plain.state.download(f))


def test_parquet_behind_the_ring_equals_the_synchronous_writer(sched, tmp_path):
    names = [("phi", "phi"), ("u", "u")]
    dt = 0.01
    a = modelc_sim(sched)
    pa_ = L.ParquetObserver(a.grid, names, 1, tmp_path / "async")
    obs = L.AsyncObserver(every=4, nslots=6, sinks=[pa_], fields=names)
    a.add_observer(obs)
    a.run(dt, 13, graph=True)
    obs.close()
    b = modelc_sim(sched)
    b.add_observer(L.ParquetObserver(b.grid, names, 4, tmp_path / "sync"))
    b.run(dt, 13)
    files = sorted(p.name for p in (tmp_path / "sync").iterdir())
    assert files == ["snap_0000001.parquet", "snap_0000004.parquet", "snap_0000008.parquet",
                     "snap_0000012.parquet", "static_0000000.parquet"]
    assert sorted(p.name for p in (tmp_path / "async").iterdir()) == files
    for name in files:
        assert pq.read_table(tmp_path / "async" / name).equals(pq.read_table(tmp_path / "sync" / name)), name


def test_parquet_follows_an_amr_run_through_its_regrids(sched, tmp_path):
    # the reference's grid-aware path: every level's blocks with their level
    # and patch per cell, the static file of the snapshot's epoch, snapshot
    # rows equal to the hierarchy's interiors at their step
    def make():
        base = L.CartesianGrid([32, 32], [8, 8], [0.0, 0.0], [H, H])
        grid = L.AmrGrid.from_patches(base, [2], [])
        model = L.ModelC(0.06, 3.19, 0.0)
        adapt = L.BergerOliger(L.GradientTagger("phi", 0.05), L.RegridPolicy(4, 1, L.ClusterParams(0.7, 4)))
        sim = L.AmrSimulation(grid, L.FiniteVolume(), model, L.Subcycling(0), sched, L.CudaAllocator("f64"), adapt)
        c = 16 * H
        phi, u = sim.get("phi"), sim.get("u")
        for b in range(sim.num_blocks):
            x, y = sim.centers(b)
            phi[b][1:-1, 1:-1] = -np.tanh((np.hypot(x - c, y - c) - 2.5) / np.sqrt(2.0))
            u[b][1:-1, 1:-1] = -0.7
        sim.set("phi", phi)
        sim.set("u", u)
        return sim

    names = [("phi", "phi"), ("u", "u")]
    twin = make()
    dt = twin.stable_dt()
    want = {}
    for k in range(1, 11):
        twin.run(dt, 1)
        if k == 1 or k % 3 == 0:
            x = np.concatenate([twin.centers(b)[0].reshape(-1) for b in range(twin.num_blocks)])
            want[k] = (twin.epoch, {n: np.concatenate([s[1:-1, 1:-1].reshape(-1) for s in twin.get(f)])
                                    for n, f in names}, x, twin.patches())
    sim = make()
    sim.add_observer(L.ParquetObserver(sim.grid, names, 3, tmp_path))
    sim.run(dt, 10)
    # the hierarchy was refined before the first snapshot (the writer's
    # epoch changes are covered on the host, test_observe.py)
    assert any(l > 0 for l, _, _ in want[1][3])
    for k, (epoch, cols, x, patches) in want.items():
        snap = pq.read_table(tmp_path / f"snap_{k:07d}.parquet")
        assert np.array_equal(snap["epoch"].to_numpy(), np.full(len(x), epoch, dtype=np.int64))
        for n, _ in names:
            assert np.array_equal(snap[n].to_numpy(), cols[n]), (k, n)
        st = pq.read_table(tmp_path / f"static_{epoch:07d}.parquet")
        assert np.array_equal(st["x"].to_numpy(), x)
        lv = np.concatenate([np.full((hi[0] - lo[0]) * (hi[1] - lo[1]), float(l)) for l, lo, hi in patches])
        assert np.array_equal(st["level"].to_numpy(), lv)
