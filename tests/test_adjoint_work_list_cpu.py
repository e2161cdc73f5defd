"""The counting rule behind the adjoint strip kernel's work list, on the CPU.

Each warp of a grid of W warps runs unit w first, then takes
n = counter++ - base and runs unit W + n while that is below the launch's U
units (lg_adjoint.cu, adjoint_strip_kernel).  The host passes base = the
units of the launches before (lg_ensemble.cu, value_and_grad), which holds
only if every launch advances the counter by exactly U whatever order the
warps finish in: one successful take per unit past the first wave and one
failing take per warp that ran a unit.  This simulates that protocol with
random finishing orders and checks the rule and that every unit runs once.
"""
import random

import pytest


def run_launch(counter, base, warps, units, rng):
    """One launch; returns (new counter, units in the order they ran)."""
    ran = []
    # the warps whose first unit exists, each with the time it finishes that unit
    active = [(rng.random(), w) for w in range(min(warps, units))]
    for _, w in active:
        ran.append(w)
    while active:
        active.sort()
        t, w = active.pop(0)  # the next warp to finish takes from the list
        n = counter - base
        counter += 1
        unit = warps + n if 0 <= n < units else units  # a wrapped value would end the warp too
        if unit < units:
            ran.append(unit)
            active.append((t + rng.random(), w))
    return counter, ran


@pytest.mark.parametrize("warps,units", [(2368, 4608), (2368, 9216), (2368, 2304), (8, 8), (8, 9), (16, 1), (5, 0)])
def test_each_launch_advances_the_counter_by_its_units(warps, units):
    rng = random.Random(warps * 7919 + units)
    counter = 0
    for launch in range(4):
        base = launch * units
        assert counter == base
        counter, ran = run_launch(counter, base, warps, units, rng)
        assert sorted(ran) == list(range(units))  # every unit once, none skipped
    assert counter == 4 * units


def test_a_wrong_base_skips_units():
    # the failure the base guards against: a base above the counter makes
    # every take fail, so only the first wave runs
    rng = random.Random(1)
    _, ran = run_launch(0, 10**6, 4, 20, rng)
    assert sorted(ran) == [0, 1, 2, 3]
