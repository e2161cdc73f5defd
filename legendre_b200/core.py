"""Scheduler, allocator, state and simulation: the host side of the device path.

These mirror the reference's seams one to one:

* :class:`CudaScheduler` -- the type-level selector of the device path, in
  the slot of ``SerialScheduler``/``RayonScheduler``
  (src/core/scheduler.rs:25-84).  It owns one CUDA stream (an ``lg_ctx``).
* :class:`CudaAllocator` -- the ``Allocator`` (src/core/storage.rs:148-154)
  handing out one device arena per state, block-major slabs, zero
  initialised, in FP64 or FP32.
* :class:`StateBuilder` / :class:`DeviceState` -- ``StateBuilder`` and
  ``State`` (src/core/state.rs:135-296): named fields with ghost widths and
  driver incidence, slabs in the reference's layout.
* :class:`Simulation` -- ``Simulation`` (src/core/simulation.rs:69-299): owns
  grid, model, integrator, scheduler and state; ``step(dt)`` runs one
  integrator step on the device.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _native as N

TIME = "time"


def wiener(j: int = 0):
    """The j-th Wiener driver (src/core/driver.rs:115-129)."""
    return ("wiener", int(j))


class CudaScheduler:
    """One CUDA device and stream; every kernel of the path runs in order on it."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        h = C.c_void_p()
        N.check(N.lib.lg_ctx_create(int(device), C.c_void_p(stream) if stream else None, C.byref(h)))
        self.handle = h
        self.device = device
        self._owned = []

    def _own(self, destroy):
        self._owned.append(destroy)

    def sync(self, timeout_ms: int = -1) -> None:
        N.check(N.lib.lg_sync(self.handle, int(timeout_ms)), self.handle)

    @property
    def kernel_launches(self) -> int:
        """Kernels this scheduler has launched (its own kernels only)."""
        return int(N.lib.lg_ctx_kernel_launches(self.handle))

    def max_concurrency(self) -> int:
        return 1

    def compute_peaks(self) -> dict:
        """Measured FP64/FP32 FMA, integer multiply-add and ALU operation
        rates of this device (operations per second over all SMs), the
        compute-side roofline denominators of the step kernels."""
        out = N.ComputePeaks()
        N.check(N.lib.lg_measure_compute_peaks(self.handle, C.byref(out)), self.handle)
        return {"dfma_per_s": out.dfma_per_s, "ffma_per_s": out.ffma_per_s, "imad_per_s": out.imad_per_s,
                "alu_per_s": out.alu_per_s, "sms": out.sms, "clock_mhz": out.clock_mhz}

    def close(self) -> None:
        if self.handle:
            for destroy in reversed(self._owned):
                destroy()
            self._owned.clear()
            N.lib.lg_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class CudaAllocator:
    """Device allocator: ``dtype`` is ``"f64"`` (the reference's arithmetic) or ``"f32"``."""

    dtype: str = "f64"

    def __post_init__(self):
        if self.dtype not in ("f64", "f32"):
            raise ValueError("dtype must be 'f64' or 'f32'")

    @property
    def code(self) -> int:
        return N.LG_F64 if self.dtype == "f64" else N.LG_F32

    @property
    def numpy_dtype(self):
        return np.float64 if self.dtype == "f64" else np.float32


@dataclass
class FieldSpec:
    """A registered field (src/core/state.rs:75-102)."""

    name: str
    ghost: int
    drivers: List = field(default_factory=lambda: [TIME])

    def is_static(self) -> bool:
        return not self.drivers


class StateBuilder:
    """Collects field registrations before allocation (state.rs:135-216)."""

    def __init__(self):
        self.specs: List[FieldSpec] = []

    def register(self, name: str, ghost: int) -> int:
        return self._push(FieldSpec(name, int(ghost), [TIME]))

    def register_driven(self, name: str, ghost: int, drivers: Sequence) -> int:
        return self._push(FieldSpec(name, int(ghost), list(drivers)))

    def register_static(self, name: str, ghost: int) -> int:
        return self._push(FieldSpec(name, int(ghost), []))

    def _push(self, spec: FieldSpec) -> int:
        self.specs.append(spec)
        return len(self.specs) - 1

    def build(self, grid, scheduler: CudaScheduler, alloc: CudaAllocator) -> "DeviceState":
        return DeviceState(grid, scheduler, alloc, self.specs)


class DeviceState:
    """Device-resident block-major state (the reference's ``State``)."""

    def __init__(self, grid, scheduler: CudaScheduler, alloc: CudaAllocator, specs: Sequence[FieldSpec]):
        self.grid = grid
        self.scheduler = scheduler
        self.alloc = alloc
        self.specs = list(specs)
        nf = len(self.specs)
        ghosts = (C.c_int * nf)(*[s.ghost for s in self.specs])
        h = C.c_void_p()
        N.check(N.lib.lg_state_create(scheduler.handle, grid.device(scheduler), alloc.code, nf, ghosts, C.byref(h)),
                scheduler.handle)
        self.handle = h
        scheduler._own(self._destroy)

    def _destroy(self):
        if self.handle:
            N.lib.lg_state_destroy(self.handle)
            self.handle = None

    # ---------------------------------------------------------------- fields
    def field(self, name: str) -> Optional[int]:
        """Handle (index) of the field registered under ``name`` (state.rs:373-386)."""
        for i, s in enumerate(self.specs):
            if s.name == name:
                return i
        return None

    def _index(self, f) -> int:
        i = self.field(f) if isinstance(f, str) else int(f)
        if i is None or not 0 <= i < len(self.specs):
            raise KeyError(f)
        return i

    def slab_shape(self, f):
        g = self.specs[self._index(f)].ghost
        return tuple(b + 2 * g for b in reversed(self.grid.block_cells))

    def download(self, f) -> np.ndarray:
        """All slabs of field ``f``: array (num_blocks, *reversed(ghosted dims)),
        i.e. ``[block][..., j, i]`` with dimension 0 fastest."""
        i = self._index(f)
        nb = self.grid.num_blocks()
        out = np.empty((nb,) + self.slab_shape(i), dtype=self.alloc.numpy_dtype)
        N.check(N.lib.lg_state_download_field(self.handle, i, out.ctypes.data_as(C.c_void_p), out.size),
                self.scheduler.handle)
        return out

    def upload(self, f, data) -> None:
        i = self._index(f)
        arr = np.ascontiguousarray(data, dtype=self.alloc.numpy_dtype)
        expect = self.grid.num_blocks() * self.grid.block_len(self.specs[i].ghost)
        if arr.size != expect:
            raise ValueError(f"field {f!r}: expected {expect} elements, got {arr.size}")
        N.check(N.lib.lg_state_upload_field(self.handle, i, arr.ctypes.data_as(C.c_void_p), arr.size),
                self.scheduler.handle)

    def interior(self, f) -> np.ndarray:
        """Interior entries of every block: (num_blocks, *reversed(block_cells))."""
        g = self.specs[self._index(f)].ghost
        a = self.download(f)
        sl = (slice(None),) + tuple(slice(g, g + n) for n in reversed(self.grid.block_cells))
        return np.ascontiguousarray(a[sl])

    def field_sum(self, f) -> float:
        """FP64 sum of field ``f`` over every block's interior cells, on the
        device in a fixed order (the same state gives the same bits)."""
        out = C.c_double()
        N.check(N.lib.lg_state_field_sum(self.handle, self._index(f), C.byref(out)), self.scheduler.handle)
        return out.value

    def fill_ghosts(self, f) -> None:
        """``fill_ghosts_mirror`` for one field (cartesian.rs:392-401)."""
        N.check(N.lib.lg_fill_ghosts(self.handle, self._index(f)), self.scheduler.handle)

    def slab_pointer(self, block: int, f):
        """Device address and length of one slab (``as_slice`` on device memory)."""
        p, n = C.c_void_p(), C.c_int64()
        N.check(N.lib.lg_state_slab(self.handle, int(block), self._index(f), C.byref(p), C.byref(n)),
                self.scheduler.handle)
        return p.value, n.value

    @property
    def time(self):
        t, s = C.c_double(), C.c_int64()
        N.check(N.lib.lg_state_get_time(self.handle, C.byref(t), C.byref(s)))
        return t.value, s.value

    def set_time(self, t: float, step_index: int = 0) -> None:
        N.check(N.lib.lg_state_set_time(self.handle, float(t), int(step_index)))


def observed_stretches(k: int, nsteps: int, everys) -> List[int]:
    """Lengths of the runs between observations: starting after step k,
    ``nsteps`` steps cut after every step that an observer with one of the
    cadences ``everys`` fires on (step 1 and multiples of its cadence)."""
    from .observe import fires

    out, done = [], 0
    while done < nsteps:
        stop = nsteps - done
        for s in range(1, stop + 1):
            if any(fires(k + done + s, e) for e in everys):
                stop = s
                break
        out.append(stop)
        done += stop
    return out


class Simulation:
    """Sole owner of grid, discretization, model, integrator, scheduler and state.

    ``step(dt)`` mirrors ``Simulation::step`` (simulation.rs:255-290) for the
    non-adaptive policy: one integrator step on the device, then ``t += dt``.
    ``run(dt, n)`` performs n such steps in one call (optionally replayed
    from a captured CUDA graph); results are identical to n ``step`` calls.
    """

    def __init__(self, grid, disc, model, integrator, scheduler: CudaScheduler, alloc: CudaAllocator):
        builder = StateBuilder()
        model.register_fields(builder)
        # simulation.rs:149-160: every declared stochastic driver moves a field
        for drv in model.stochastic_drivers():
            if not any(drv in spec.drivers for spec in builder.specs):
                raise ValueError(f"model declares stochastic driver {drv} but no field is driven by it")
        self.grid = grid
        self.disc = disc
        self.model = model
        self.integrator = integrator
        self.scheduler = scheduler
        self.alloc = alloc
        self.state = builder.build(grid, scheduler, alloc)
        integrator.validate(model, grid, disc)
        self.observers = []

    def stable_dt(self) -> Optional[float]:
        return self.integrator.suggested_dt(self.model, self.grid)

    def time(self) -> float:
        return self.state.time[0]

    def step_index(self) -> int:
        return self.state.time[1]

    def step(self, dt: float) -> None:
        self.run(dt, 1)

    def add_observer(self, observer) -> None:
        """Observers are called after the steps they fire on (step 1 and every
        ``observer.every`` steps) with (step, t, epoch, grid, state), as
        ``Simulation::step`` notifies them (simulation.rs:286-289)."""
        self.observers.append(observer)

    def run(self, dt: float, nsteps: int, graph: bool = False, variant: int = 0) -> None:
        nsteps = int(nsteps)
        if not self.observers:
            self.integrator.run(self, float(dt), nsteps, graph=graph, variant=variant)
            return
        # run in stretches that end on the steps some observer fires on
        for stop in observed_stretches(self.step_index(), nsteps, [getattr(o, "every", 1) for o in self.observers]):
            self.integrator.run(self, float(dt), stop, graph=graph, variant=variant)
            step = self.step_index()
            for o in self.observers:
                o.observe(step, self.time(), 0, self.grid, self.state)

    def value_and_grad(self, dt: float, nsteps: int, ckpt_every: int, target, cell_grads: bool = True) -> dict:
        """The backward API of this Simulation: from its current state, runs
        ``nsteps`` Euler-Maruyama steps of Model C (the trajectory ``run``
        gives), evaluates L = sum over the cells of (phi_T - target)^2 and
        returns L with dL/d(lambda, D, eps4, Delta) and, with ``cell_grads``,
        dL/dphi_0 and dL/du_0 per cell -- the hand-written adjoint of the fused
        step with a checkpoint every ``ckpt_every`` steps (the noise replays
        from its keys).  Delta shifts the initial u by -Delta on every cell.
        ``target`` and the cell gradients are (cells_y, cells_x) arrays.  The
        state is left at the final step, as after ``run``.  2-D zero-flux
        Model C grids, axis-aligned, only."""
        import numpy as np

        from .integrators import EulerMaruyama
        from .physics import ModelC

        if not isinstance(self.model, ModelC) or not isinstance(self.integrator, EulerMaruyama):
            raise TypeError("value_and_grad differentiates Model C stepped by EulerMaruyama")
        shape = (self.grid.cells[1], self.grid.cells[0])
        tgt = np.ascontiguousarray(np.broadcast_to(target, shape), dtype=np.float64)
        loss, gp = np.empty(1), np.empty(4)
        dphi = np.empty(shape) if cell_grads else None
        du = np.empty(shape) if cell_grads else None
        ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None
        p = self.model.params(flux_tol=self.disc.tol)
        N.check(N.lib.lg_modelc_value_and_grad(self.state.handle, C.byref(p), float(dt),
                                               int(self.integrator.seed) & ((1 << 64) - 1), int(nsteps),
                                               int(ckpt_every), ptr(tgt), ptr(loss), ptr(gp), ptr(dphi), ptr(du)),
                self.scheduler.handle)
        return {"loss": float(loss[0]), "lambda": float(gp[0]), "d_thermal": float(gp[1]), "eps4": float(gp[2]),
                "delta": float(gp[3]), "phi0": dphi, "u0": du}

    def autotune(self, dt: float, trial_steps: int = 20):
        """Pick the fastest Model C step variant for this grid and precision by
        timing every candidate from a copy of the state (the state, its time
        and step index are left as they were); later ``run`` calls with the
        default variant use it.  Returns (variant, ms per step)."""
        from .integrators import EulerMaruyama
        from .physics import ModelC

        if not isinstance(self.model, ModelC):
            raise TypeError("the autotuner covers the Model C step")
        seed = self.integrator.seed if isinstance(self.integrator, EulerMaruyama) else 0
        p = self.model.params(flux_tol=self.disc.tol)
        v, ms = C.c_int(), C.c_double()
        N.check(N.lib.lg_modelc_autotune(self.state.handle, C.byref(p), float(dt), int(seed) & ((1 << 64) - 1),
                                         int(trial_steps), C.byref(v), C.byref(ms)), self.scheduler.handle)
        return v.value, ms.value
