"""Small helpers shared by the tests (no product code)."""
from __future__ import annotations

import numpy as np


def relative_eq(a, b, max_relative, epsilon):
    """approx::relative_eq semantics, elementwise."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    diff = np.abs(a - b)
    return (a == b) | (diff <= epsilon) | (diff <= np.maximum(np.abs(a), np.abs(b)) * max_relative)


def centers(cells, block, origin, spacing, d):
    """Cell-centre coordinate along d for every interior cell, shaped
    (num_blocks, *reversed(block)) -- CartesianGrid::cell_center
    (cartesian.rs:588-597).  The product (g + i + 0.5) * h must be exact in
    binary64 for the result to equal the reference's fma; true for the grids
    used in the tests (origin 0 makes it exact unconditionally)."""
    D = len(cells)
    nb = [c // b for c, b in zip(cells, block)]
    nblocks = int(np.prod(nb))
    out = np.empty((nblocks,) + tuple(reversed(block)), dtype=np.float64)
    for b in range(nblocks):
        rem, coords = b, []
        for k in range(D):
            coords.append(rem % nb[k])
            rem //= nb[k]
        i = np.arange(block[d], dtype=np.float64)
        a = (float(coords[d] * block[d]) + i) + 0.5
        x = a * spacing[d] + origin[d] if origin[d] != 0.0 else a * spacing[d]
        shape = [1] * D
        shape[D - 1 - d] = block[d]
        out[b] = np.broadcast_to(x.reshape(shape), tuple(reversed(block)))
    return out


def with_ghosts(interior, ghost):
    """Embed interior arrays (num_blocks, ...) into zeroed ghost-inclusive slabs."""
    nb = interior.shape[0]
    shape = (nb,) + tuple(n + 2 * ghost for n in interior.shape[1:])
    out = np.zeros(shape, dtype=interior.dtype)
    sl = (slice(None),) + tuple(slice(ghost, ghost + n) for n in interior.shape[1:])
    out[sl] = interior
    return out
