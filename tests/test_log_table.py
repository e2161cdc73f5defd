"""The FP64 Box-Muller logarithm's table (legendre_b200/csrc/lg_log_table.h)
against its generator, and the reduction it serves restated on the CPU.

The device logarithm (log_unit_interval, lg_common.cuh) computes
ln u = e ln 2 + L_j + log1p(f invF_j - 1); the restatement below follows it
operation for operation (math.fma) and is compared with the exact logarithm
(a 40-digit decimal one) on the arguments where the reduction is most
fragile: u next to 1, the smallest u, both sides of sqrt(2) and the edges of
the table's bins.
"""
import math
import random
import sys
from decimal import Decimal, getcontext
from pathlib import Path

CSRC = Path(__file__).resolve().parents[1] / "legendre_b200" / "csrc"
sys.path.insert(0, str(CSRC))
import gen_log_table  # noqa: E402


def test_header_is_the_generator_output():
    assert (CSRC / "lg_log_table.h").read_text() == gen_log_table.render()


def test_table_entries():
    getcontext().prec = 40
    ent = gen_log_table.entries()
    assert len(ent) == gen_log_table.J_MAX - gen_log_table.J_MIN + 1 == 91
    for j, inv, lj in ent:
        assert inv == 128.0 / (128 + j)  # the correctly rounded reciprocal of F_j
        if j == 0:
            assert inv == 1.0 and lj == 0.0 and math.copysign(1.0, lj) == 1.0
        exact = -Decimal(inv).ln()
        assert abs(Decimal(lj) - exact) <= abs(exact) * Decimal(2) ** -53


def _fma(a, b, c):
    # exact product and sum, one rounding (math.fma where the interpreter has it)
    if hasattr(math, "fma"):
        return math.fma(a, b, c)
    from fractions import Fraction
    return float(Fraction(a) * Fraction(b) + Fraction(c))


_TABLE = {}


def _log_unit_interval(u):
    if not _TABLE:
        _TABLE.update({j: (inv, lj) for j, inv, lj in gen_log_table.entries()})
    table = _TABLE
    m, e = math.frexp(u)          # u = m 2^e, m in [0.5, 1)
    f, e = 2.0 * m, e - 1         # f in [1, 2)
    if f > 1.4142135623730951:
        f, e = 0.5 * f, e + 1
    j = round((f - 1.0) * 128.0)  # ties to even, as __double2int_rn
    inv, lj = table[j]
    r = _fma(f, inv, -1.0)
    q = 1.0 / 7.0
    for c in (-1.0 / 6.0, 1.0 / 5.0, -0.25, 1.0 / 3.0, -0.5):
        q = _fma(q, r, c)
    p = _fma(r * r, q, r)
    ln2_hi, ln2_lo = float.fromhex("0x1.62e42fefa3800p-1"), float.fromhex("0x1.ef35793c76730p-45")
    return _fma(float(e), ln2_hi, lj) + _fma(float(e), ln2_lo, p)


def _rel(u):
    got = _log_unit_interval(u)
    exact = Decimal(u).ln()
    if exact == 0:
        return abs(got)
    return float(abs((Decimal(got) - exact) / exact))


def test_reduction_within_4e16_of_the_exact_logarithm():
    getcontext().prec = 40
    rng = random.Random(5)
    us = [1.0]
    us += [1.0 - m * 2.0 ** -53 for m in range(1, 400)]                       # ln u tiny
    us += [m * 2.0 ** -53 for m in range(1, 400)]                             # the smallest u
    us += [math.ldexp(1.4142135623730951 + d * 2.0 ** -52, ex) for d in range(-30, 30) for ex in (-1, -7, -40)]
    us += [math.ldexp(1.0 + (j + 0.5) / 128 + d * 2.0 ** -52, ex)            # bin edges
           for j in range(-38, 55) for d in (-2, -1, 0, 1, 2) for ex in (-1, -2, -30)]
    us += [((rng.getrandbits(53)) + 1) * 2.0 ** -53 for _ in range(3000)]     # the uniforms
    us = [u for u in us if 2.0 ** -53 <= u <= 1.0]
    assert _log_unit_interval(1.0) == 0.0 and math.copysign(1.0, _log_unit_interval(1.0)) == 1.0
    worst = max(_rel(u) for u in us)
    assert worst <= 4e-16, worst
