"""Seed placement of the reference's Model C example, in pure Python.

Nothing here touches the device library, so a CPU-only caller (the timed
CPU baseline, for instance) can place grains without loading
``liblegendre_b200.so``.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Sequence

from .rng import fma


@dataclass
class Grain:
    """One nucleation site (phasefield.rs:78-88)."""

    center: Sequence[float]
    radius: float
    orientation: float = 0.0


def seed_positions(cells: int, h: float, nseeds: int, seed: int, radius: Optional[float] = None,
                   orient: bool = False):
    """Seed placement of the model_c example (examples/model_c.rs:175-206):
    one corner seed, or ``nseeds`` uniform positions with a margin of two
    radii; with ``orient`` grain i has the orientation
    unit_open(mix_key(seed, [i, 2])) * pi/2 (the 4-fold fundamental domain)."""
    import math

    from .rng import mix_key, unit_open

    radius = 10.0 * h if radius is None else float(radius)
    orientation = (lambda i: unit_open(mix_key(seed, [i, 2])) * (math.pi / 2)) if orient else (lambda i: 0.0)
    if nseeds <= 1:
        return [Grain((h, h), radius, orientation(0))]
    extent = cells * h
    margin = 2.0 * radius
    span = fma(2.0, -margin, extent)
    out = []
    for i in range(nseeds):
        x = margin + unit_open(mix_key(seed, [i, 0])) * span
        y = margin + unit_open(mix_key(seed, [i, 1])) * span
        out.append(Grain((x, y), radius, orientation(i)))
    return out
