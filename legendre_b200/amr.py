"""2-D adaptive mesh refinement on the device, mirroring the reference's
``AmrGrid`` / ``BergerOliger`` / ``Subcycling`` (src/geometry/amr/*,
src/integrators/subcycling.rs) and ``Simulation::adaptive``
(src/core/simulation.rs:137-183).

The hierarchy, its transfer plans and the state live in one ``lg_amr_sim``
(C ABI); ghost fill, restriction, tagging and the per-level steps run on the
GPU, clustering and migration on the host at regrid cadence.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .geometry import GridError
from .physics import Heat, ModelC

Box = Tuple[Tuple[int, int], Tuple[int, int]]


@dataclass
class CellBox:
    """Half-open box of cells at one level (amr/cluster.rs:27-37)."""

    lo: Tuple[int, int]
    hi: Tuple[int, int]


@dataclass
class AmrGrid:
    """A patch hierarchy over a base Cartesian tiling (amr/grid.rs:55-196):
    ``base`` is a 2-D ``CartesianGrid``, ``ratios[l]`` the refinement from
    level l to l+1, ``levels[l]`` the level-(l+1) patch boxes."""

    base: object
    ratios: Sequence[int]
    levels: Sequence[Sequence[CellBox]] = field(default_factory=list)

    @classmethod
    def from_patches(cls, base, ratios, levels=()):
        """The hierarchy, validated as the reference's ``from_patches`` does
        (ratios >= 2, patches inside their level's domain, aligned to the
        ratio, disjoint and properly nested): ``GridError`` otherwise."""
        g = cls(base, list(ratios), [list(l) for l in levels])
        if base.dim == 2:  # the device AMR path is 2-D; AmrSimulation refuses other bases
            g.validate()
        return g

    def validate(self) -> None:
        pa = np.ascontiguousarray(self.patch_array())
        r = (C.c_uint32 * max(1, len(self.ratios)))(*[int(x) for x in self.ratios])
        err = C.create_string_buffer(256)
        rc = N.lib.lg_amr_check_hierarchy((C.c_int64 * 2)(*self.base.cells), (C.c_int64 * 2)(*self.base.block_cells),
                                          r, len(self.ratios), pa.ctypes.data_as(C.POINTER(C.c_int64)), len(pa),
                                          err, len(err))
        if rc != N.LG_OK:
            raise GridError(err.value.decode() or f"invalid hierarchy ({rc})")

    def patch_array(self) -> np.ndarray:
        rows = [[lv + 1, b.lo[0], b.lo[1], b.hi[0], b.hi[1]] for lv, boxes in enumerate(self.levels) for b in boxes]
        return np.array(rows, dtype=np.int64).reshape(-1, 5)


@dataclass
class ClusterParams:
    """Berger-Rigoutsos knobs (amr/cluster.rs:115-135)."""

    efficiency: float = 0.8
    min_width: int = 4


def cluster(flags, params: Optional[ClusterParams] = None) -> List[CellBox]:
    """Berger-Rigoutsos boxes covering the flagged cells of one level
    (``cluster``, amr/cluster.rs:144-290), computed by the library's host code
    (the same code as its regrids); ``flags`` is a sequence of (x, y)."""
    params = params or ClusterParams()
    arr = np.ascontiguousarray(np.asarray(flags, dtype=np.int64).reshape(-1, 2))
    cap = max(1, len(arr))  # every box holds at least one flag
    out = np.zeros((cap, 4), dtype=np.int64)
    n = C.c_int64()
    N.check(N.lib.lg_amr_cluster(arr.ctypes.data_as(C.POINTER(C.c_int64)), len(arr), float(params.efficiency),
                                 int(params.min_width), out.ctypes.data_as(C.POINTER(C.c_int64)), cap, C.byref(n)))
    return [CellBox((int(b[0]), int(b[1])), (int(b[2]), int(b[3]))) for b in out[:n.value]]


@dataclass
class GradientTagger:
    """Flag where max_d |u(i+e_d) - u(i-e_d)|/2 > threshold (adapt.rs:48-104)."""

    field: str
    threshold: float


@dataclass
class RegridPolicy:
    """Regrid cadence, buffer zone and clustering (adapt.rs:106-129)."""

    every: int = 4
    buffer: int = 2
    cluster: ClusterParams = field(default_factory=ClusterParams)


@dataclass
class BergerOliger:
    """The Berger-Oliger adaptivity policy (adapt.rs:131-237)."""

    tagger: GradientTagger
    policy: RegridPolicy


@dataclass
class Subcycling:
    """Berger-Oliger subcycled time integration (subcycling.rs:46-152)."""

    seed: int = 0


class AmrSimulation:
    """``Simulation`` on an ``AmrGrid`` (see the module docs).

    ``integrator`` is :class:`Subcycling` (per-level dt) or an
    ``EulerMaruyama``/``ForwardEuler`` (one global dt at the finest level's
    stable step).  ``adapt`` is a :class:`BergerOliger` or ``None`` (Static).
    """

    def __init__(self, grid: AmrGrid, disc, model, integrator, scheduler, alloc, adapt: Optional[BergerOliger] = None):
        from .integrators import EulerMaruyama, FiniteVolume, ForwardEuler

        if alloc.dtype != "f64":
            raise ValueError("the AMR path is FP64")
        base = grid.base
        if base.dim != 2:
            raise ValueError("the AMR path is 2-D")
        self.grid = grid
        self.observers = []
        self.model = model
        self.scheduler = scheduler
        if isinstance(model, ModelC):
            if not isinstance(disc, FiniteVolume):
                raise TypeError("Model C needs the FiniteVolume policy")
            kind, params, kappa = N.LG_MODEL_C, C.byref(model.params(flux_tol=disc.tol)), 0.0
            self.fields = ["phi", "u"]
        elif isinstance(model, Heat):
            kind, params, kappa = N.LG_MODEL_HEAT, None, model.kappa
            self.fields = ["u"]
        else:
            raise TypeError(f"no AMR device path for {type(model).__name__}")
        if isinstance(integrator, Subcycling):
            integ, seed = N.LG_AMR_SUBCYCLING, integrator.seed
        elif isinstance(integrator, (EulerMaruyama, ForwardEuler)):
            integ, seed = N.LG_AMR_GLOBAL_DT, getattr(integrator, "seed", 0)
        else:
            raise TypeError("integrator must be Subcycling, EulerMaruyama or ForwardEuler")
        pol = None
        if adapt is not None:
            fld = self.fields.index(adapt.tagger.field)
            pol = N.AmrPolicy(adapt.policy.every, adapt.policy.buffer, adapt.policy.cluster.min_width,
                              adapt.policy.cluster.efficiency, adapt.tagger.threshold, fld)
        pa = grid.patch_array()
        out = C.c_void_p()
        N.check(N.lib.lg_amr_sim_create(
            scheduler.handle, (C.c_int64 * 2)(*base.cells), (C.c_int64 * 2)(*base.block_cells),
            (C.c_double * 2)(*base.origin), (C.c_double * 2)(*base.spacing),
            (C.c_uint32 * max(1, len(grid.ratios)))(*grid.ratios), len(grid.ratios),
            pa.ctypes.data_as(C.POINTER(C.c_int64)), len(pa), kind, params, kappa, integ, int(seed) & (2**64 - 1),
            C.byref(pol) if pol is not None else None, C.byref(out)), scheduler.handle)
        self.handle = out
        scheduler._own(self._destroy)

    def _destroy(self):
        if self.handle:
            N.lib.lg_amr_sim_destroy(self.handle)
            self.handle = None

    # ----------------------------------------------------------- queries
    def info(self):
        nb, nl, ep = C.c_int64(), C.c_int(), C.c_int64()
        N.check(N.lib.lg_amr_sim_info(self.handle, C.byref(nb), C.byref(nl), C.byref(ep)))
        return nb.value, nl.value, ep.value

    @property
    def num_blocks(self):
        return self.info()[0]

    @property
    def num_levels(self):
        return self.info()[1]

    @property
    def epoch(self):
        return self.info()[2]

    def patch(self, b):
        out = (C.c_int64 * 5)()
        N.check(N.lib.lg_amr_sim_patch(self.handle, b, out))
        return int(out[0]), (int(out[1]), int(out[2])), (int(out[3]), int(out[4]))

    def patches(self):
        return [self.patch(b) for b in range(self.num_blocks)]

    def _index(self, f):
        return self.fields.index(f) if isinstance(f, str) else int(f)

    def get(self, f) -> List[np.ndarray]:
        """Per-block ghost-inclusive slabs of field f, each (ny+2, nx+2)."""
        n = C.c_int64()
        N.check(N.lib.lg_amr_sim_field_len(self.handle, C.byref(n)))
        flat = np.empty(n.value)
        N.check(N.lib.lg_amr_sim_get_field(self.handle, self._index(f), flat.ctypes.data_as(C.POINTER(C.c_double)),
                                           n.value), self.scheduler.handle)
        out, off = [], 0
        for lv, lo, hi in self.patches():
            nx, ny = hi[0] - lo[0], hi[1] - lo[1]
            k = (nx + 2) * (ny + 2)
            out.append(flat[off:off + k].reshape(ny + 2, nx + 2).copy())
            off += k
        return out

    def set(self, f, slabs) -> None:
        flat = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.float64).ravel() for s in slabs]))
        N.check(N.lib.lg_amr_sim_set_field(self.handle, self._index(f), flat.ctypes.data_as(C.POINTER(C.c_double)),
                                           flat.size), self.scheduler.handle)

    def time(self):
        t, s = C.c_double(), C.c_int64()
        N.check(N.lib.lg_amr_sim_time(self.handle, C.byref(t), C.byref(s)))
        return t.value

    def step_index(self):
        t, s = C.c_double(), C.c_int64()
        N.check(N.lib.lg_amr_sim_time(self.handle, C.byref(t), C.byref(s)))
        return s.value

    def stable_dt(self) -> float:
        dt = C.c_double()
        N.check(N.lib.lg_amr_sim_suggested_dt(self.handle, C.byref(dt)))
        return dt.value

    # ------------------------------------------------------------ steps
    def step(self, dt: float) -> None:
        self.run(dt, 1)

    def add_observer(self, observer) -> None:
        """Observers are called after the coarse steps they fire on with
        (step, t, epoch, grid, sim): the sim itself is the state they read, so
        a grid-aware observer follows regrids through the epoch."""
        self.observers.append(observer)

    def run(self, dt: float, nsteps: int, graph: bool = False, persistent: bool = False) -> None:
        """`nsteps` coarse steps.  `graph` replays pairs of coarse steps from a
        CUDA graph; `persistent` runs each pair as one cooperative launch
        (every level's fused fill + step and every restriction, separated by
        grid barriers) and takes precedence."""
        flags = (N.LG_RUN_GRAPH if graph else 0) | (N.LG_RUN_PERSISTENT if persistent else 0)
        if not self.observers:
            N.check(N.lib.lg_amr_sim_step(self.handle, float(dt), int(nsteps), flags), self.scheduler.handle)
            return
        from .core import observed_stretches

        for stop in observed_stretches(self.step_index(), int(nsteps), [getattr(o, "every", 1) for o in self.observers]):
            N.check(N.lib.lg_amr_sim_step(self.handle, float(dt), stop, flags), self.scheduler.handle)
            for o in self.observers:
                o.observe(self.step_index(), self.time(), self.epoch, self.grid, self)

    def set_barrier_spin_limit(self, polls: int) -> None:
        """Polls a grid barrier of the persistent launch waits before it gives
        up (the step then raises LegendreError with LG_ERR_TIMEOUT and the
        state is invalid); 0 makes a waiting barrier give up at once."""
        N.check(N.lib.lg_amr_sim_set_barrier_spin_limit(self.handle, int(polls)), self.scheduler.handle)

    # ------------------------------------------------------ transfers (c)
    def restrict(self, f) -> None:
        N.check(N.lib.lg_amr_restrict(self.handle, self._index(f)), self.scheduler.handle)

    def fill_ghosts(self) -> None:
        N.check(N.lib.lg_amr_fill_ghosts(self.handle), self.scheduler.handle)

    def tag_level(self, f, level: int, threshold: float):
        count = C.c_int64()
        cap = 1 << 22
        out = np.zeros(2 * cap, dtype=np.int64)
        N.check(N.lib.lg_amr_tag_level(self.handle, self._index(f), level, threshold,
                                       out.ctypes.data_as(C.POINTER(C.c_int64)), cap, C.byref(count)),
                self.scheduler.handle)
        return [tuple(out[2 * i:2 * i + 2]) for i in range(min(count.value, cap))]

    def centers(self, b):
        """Cell-centre coordinates (x, y) of block b's interior, each (ny, nx):
        fma(lo + i + 0.5, h_level, origin) (amr/grid.rs:389-395)."""
        from .rng import fma
        lv, lo, hi = self.patch(b)
        base = self.grid.base
        r = 1
        for k in range(lv):
            r *= self.grid.ratios[k]
        hs = [base.spacing[d] for d in range(2)]
        for k in range(lv):
            hs = [h / float(self.grid.ratios[k]) for h in hs]
        nx, ny = hi[0] - lo[0], hi[1] - lo[1]
        xs = np.array([fma(float(lo[0] + i) + 0.5, hs[0], base.origin[0]) for i in range(nx)])
        ys = np.array([fma(float(lo[1] + j) + 0.5, hs[1], base.origin[1]) for j in range(ny)])
        return np.broadcast_to(xs[None, :], (ny, nx)).copy(), np.broadcast_to(ys[:, None], (ny, nx)).copy()
