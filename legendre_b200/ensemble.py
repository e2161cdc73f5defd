"""Batched Model C realisations and the gradient of a terminal loss.

``Ensemble`` steps many independent instances of one 2-D Cartesian grid
(zero-flux boundaries) together on the device, each with its own eps4 and
noise seed; each instance follows the trajectory its own ``Simulation`` of
``ModelC`` with ``EulerMaruyama(seed)`` would (bit for bit in FP64).  The
reference has no batched form: it runs one ``Simulation`` per realisation.

``Ensemble.value_and_grad`` is the backward API: for L_i = sum over cells of
(phi_T - target)^2 it returns dL_i/d(lambda, D, eps4, Delta) and dL_i/dphi_0,
dL_i/du_0, from a hand-written adjoint of the fused step with checkpoints
every K steps (segments recomputed, noise replayed from its counter keys).
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _native as N
from .geometry import CartesianGrid
from .physics import ModelC


class Ensemble:
    def __init__(self, grid: CartesianGrid, model: ModelC, eps4: Sequence[float], seeds: Sequence[int], scheduler,
                 dtype: str = "f64", flux_tol: float = 1e-8):
        if len(grid.cells) != 2 or any(grid.periodic):
            raise ValueError("an ensemble is a batch of non-periodic 2-D grids")
        eps4 = np.ascontiguousarray(eps4, dtype=np.float64)
        seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        if eps4.shape != seeds.shape or eps4.ndim != 1 or eps4.size == 0:
            raise ValueError("eps4 and seeds need one entry per instance")
        if dtype not in ("f64", "f32"):
            raise ValueError("dtype is 'f64' or 'f32'")
        self.grid, self.model, self.scheduler = grid, model, scheduler
        self.ninst = int(eps4.size)
        self.eps4, self.seeds = eps4, seeds
        self.dtype = dtype
        self.shape = (self.ninst, grid.cells[1], grid.cells[0])
        cells = (C.c_int64 * 2)(*grid.cells)
        block = (C.c_int64 * 2)(*grid.block_cells)
        spacing = (C.c_double * 2)(*grid.spacing)
        h = C.c_void_p()
        N.check(N.lib.lg_ensemble_create(scheduler.handle, cells, block, spacing, self.ninst,
                                         C.byref(model.params(flux_tol)),
                                         eps4.ctypes.data_as(C.POINTER(C.c_double)),
                                         seeds.ctypes.data_as(C.POINTER(C.c_uint64)),
                                         N.LG_F64 if dtype == "f64" else N.LG_F32, C.byref(h)), scheduler.handle)
        self.handle = h
        scheduler._own(self._destroy)

    def _destroy(self):
        if self.handle:
            N.lib.lg_ensemble_destroy(self.handle)
            self.handle = None

    @staticmethod
    def _field(f) -> int:
        return {"phi": 0, "u": 1, 0: 0, 1: 1}[f]

    def set(self, f, values) -> None:
        """Field ``f`` of every instance: an array (instances, ny, nx)."""
        a = np.ascontiguousarray(np.broadcast_to(values, self.shape), dtype=np.float64)
        N.check(N.lib.lg_ensemble_upload(self.handle, self._field(f), a.ctypes.data_as(C.POINTER(C.c_double)), a.size),
                self.scheduler.handle)

    def get(self, f) -> np.ndarray:
        a = np.empty(self.shape, dtype=np.float64)
        N.check(N.lib.lg_ensemble_download(self.handle, self._field(f), a.ctypes.data_as(C.POINTER(C.c_double)),
                                           a.size), self.scheduler.handle)
        return a

    def time(self):
        t, k = C.c_double(), C.c_int64()
        N.check(N.lib.lg_ensemble_get_time(self.handle, C.byref(t), C.byref(k)))
        return t.value, k.value

    def set_time(self, t: float, step_index: int = 0) -> None:
        N.check(N.lib.lg_ensemble_set_time(self.handle, float(t), int(step_index)))

    def run(self, dt: float, nsteps: int, graph: bool = False) -> None:
        N.check(N.lib.lg_ensemble_run(self.handle, float(dt), int(nsteps), N.LG_RUN_GRAPH if graph else 0),
                self.scheduler.handle)

    ADJOINT_KERNELS = {"strip": 0, "tile": 1}

    def value_and_grad(self, dt: float, nsteps: int, ckpt_every: int, target, cell_grads: bool = True,
                       kernel: str = "strip", resident_bytes: int = 0) -> dict:
        """Loss and gradients of every instance (see the module docstring); the
        state is left at the final step.  ``kernel`` picks the form of the
        step adjoint: "strip" (warps walking up the rows) or "tile"
        (shared-memory tiles); they agree up to rounding.  With
        ``resident_bytes`` > 0 the last segments whose states fit in that many
        device bytes keep them from the forward pass instead of recomputing
        them (same results, less work)."""
        if kernel not in self.ADJOINT_KERNELS:
            raise ValueError("kernel is 'strip' or 'tile'")
        N.check(N.lib.lg_ensemble_set_adjoint_kernel(self.handle, self.ADJOINT_KERNELS[kernel]), self.scheduler.handle)
        N.check(N.lib.lg_ensemble_set_resident_budget(self.handle, int(resident_bytes)), self.scheduler.handle)
        tgt = np.ascontiguousarray(np.broadcast_to(target, self.shape), dtype=np.float64)
        loss = np.empty(self.ninst)
        gp = np.empty((self.ninst, 4))
        dphi = np.empty(self.shape) if cell_grads else None
        du = np.empty(self.shape) if cell_grads else None
        ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None
        N.check(N.lib.lg_ensemble_value_and_grad(self.handle, float(dt), int(nsteps), int(ckpt_every), ptr(tgt),
                                                 ptr(loss), ptr(gp), ptr(dphi), ptr(du)), self.scheduler.handle)
        return {"loss": loss, "lambda": gp[:, 0], "d_thermal": gp[:, 1], "eps4": gp[:, 2], "delta": gp[:, 3],
                "phi0": dphi, "u0": du}
