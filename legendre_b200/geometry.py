"""Host-side grid description, mirroring the reference's ``CartesianGrid<D>``.

The grid itself is pure topology and geometry (src/geometry/cartesian.rs:28-187);
its device form -- the block-topology table the kernels read -- is created
per scheduler by :meth:`CartesianGrid.device`.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Sequence

from . import _native as N
from .rng import fma


class GridError(ValueError):
    """Invalid grid construction (the reference's ``GridError``)."""


@dataclass
class CartesianGrid:
    """Uniform Cartesian grid of ``cells`` tiled by congruent blocks.

    Mirrors ``CartesianGrid::new`` (src/geometry/cartesian.rs:48-82): every
    dimension non-empty, ``cells[d] % block_cells[d] == 0``, positive finite
    spacing.  Slabs are dimension-0-fastest with a ghost ring.
    """

    cells: Sequence[int]
    block_cells: Sequence[int]
    origin: Sequence[float]
    spacing: Sequence[float]
    periodic: Sequence[bool] = None
    _dev: dict = field(default_factory=dict, repr=False, compare=False)

    def __post_init__(self):
        self.cells = tuple(int(c) for c in self.cells)
        self.block_cells = tuple(int(c) for c in self.block_cells)
        self.origin = tuple(float(o) for o in self.origin)
        self.spacing = tuple(float(h) for h in self.spacing)
        D = len(self.cells)
        if not 1 <= D <= 3 or not (len(self.block_cells) == len(self.origin) == len(self.spacing) == D):
            raise GridError("cells, block_cells, origin and spacing must share a dimension in 1..3")
        for d in range(D):
            if not (self.cells[d] > 0 and self.block_cells[d] > 0):
                raise GridError(f"empty dimension {d}")
            if self.cells[d] % self.block_cells[d] != 0:
                raise GridError(f"dimension {d}: {self.cells[d]} cells not divisible by {self.block_cells[d]}")
            if not (self.spacing[d] > 0.0 and math.isfinite(self.spacing[d])):
                raise GridError(f"dimension {d}: invalid spacing {self.spacing[d]}")
        self.periodic = tuple(bool(p) for p in (self.periodic or (False,) * D))

    # ------------------------------------------------------------ queries
    @classmethod
    def single_block(cls, cells, origin, spacing):
        """Whole domain as one block (cartesian.rs:110-116)."""
        return cls(cells, cells, origin, spacing)

    def with_periodic(self, periodic) -> "CartesianGrid":
        """Mark dimensions periodic (cartesian.rs:94-97)."""
        return CartesianGrid(self.cells, self.block_cells, self.origin, self.spacing, tuple(periodic))

    @property
    def dim(self) -> int:
        return len(self.cells)

    @property
    def blocks_per_dim(self):
        return tuple(c // b for c, b in zip(self.cells, self.block_cells))

    def num_blocks(self) -> int:
        return math.prod(self.blocks_per_dim)

    def block_len(self, ghost: int) -> int:
        return math.prod(b + 2 * ghost for b in self.block_cells)

    def block_coords(self, block: int):
        rem, out = block, []
        for nb in self.blocks_per_dim:
            out.append(rem % nb)
            rem //= nb
        return tuple(out)

    def face_neighbor(self, block: int, dim: int, direction: int):
        """Neighbour across face (dim, +-1), wrapped in periodic dimensions; None
        at a physical boundary (cartesian.rs:162-181)."""
        c = list(self.block_coords(block))
        nb = self.blocks_per_dim
        stepped = c[dim] + (1 if direction > 0 else -1)
        if 0 <= stepped < nb[dim]:
            c[dim] = stepped
        elif self.periodic[dim]:
            c[dim] = stepped % nb[dim]
        else:
            return None
        out, stride = 0, 1
        for d in range(self.dim):
            out += c[d] * stride
            stride *= nb[d]
        return out

    def cell_center(self, block: int, idx):
        """Cell-centre coordinate (cartesian.rs:588-597): fma(global + i + 0.5, h, origin)."""
        c = self.block_coords(block)
        return tuple(
            fma((float(c[d] * self.block_cells[d]) + float(idx[d])) + 0.5, self.spacing[d], self.origin[d])
            for d in range(self.dim))

    # ------------------------------------------------------------ device
    def device(self, scheduler) -> C.c_void_p:
        """The device block-topology table of this grid on ``scheduler``."""
        key = id(scheduler)
        h = self._dev.get(key)
        if h is None:
            D = self.dim
            out = C.c_void_p()
            N.check(N.lib.lg_grid_create_cartesian(
                scheduler.handle, D, (C.c_int64 * D)(*self.cells), (C.c_int64 * D)(*self.block_cells),
                (C.c_double * D)(*self.origin), (C.c_double * D)(*self.spacing),
                (C.c_int * D)(*[int(p) for p in self.periodic]), C.byref(out)), scheduler.handle)
            h = out
            self._dev[key] = h
            scheduler._own(lambda h=h: N.lib.lg_grid_destroy(h))
        return h
