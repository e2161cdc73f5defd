"""Host-side counter-based generator of the reference (src/util/rng.rs:13-49).

Used on the host for seed placement and keys; the device generator lives in
csrc/lg_common.cuh.  Pure integer arithmetic, so both sides agree bit for bit.
"""
from __future__ import annotations

from fractions import Fraction

MASK = (1 << 64) - 1


def splitmix64(z: int) -> int:
    """SplitMix64 finalizer (rng.rs:13-18)."""
    z = (z + 0x9E3779B97F4A7C15) & MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def mix_key(seed: int, parts) -> int:
    """Chain-mix key components (rng.rs:23-29)."""
    s = splitmix64(seed & MASK)
    for p in parts:
        s = splitmix64(s ^ (p & MASK))
    return s


def unit_open(bits: int) -> float:
    """Uniform deviate in (0, 1] from 53 bits (rng.rs:35-37); exact in binary64."""
    return float((bits >> 11) + 1) * (1.0 / 9007199254740992.0)


def fma(a: float, b: float, c: float) -> float:
    """Correctly rounded a*b+c (the reference's ``f64::mul_add``)."""
    return float(Fraction(a) * Fraction(b) + Fraction(c))
