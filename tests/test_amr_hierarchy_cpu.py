"""AmrGrid.from_patches validation (lg_amr_check_hierarchy: the check the
library's AMR simulation and regrids run) against the reference's error
paths (amr/grid.rs:90-196) and the oracle's verdicts, on the CPU."""
import numpy as np
import pytest

import legendre_b200 as L
from legendre_b200.amr import AmrGrid, CellBox


def base(cells=(8, 8), block=(8, 8)):
    return L.CartesianGrid(list(cells), list(block), [0.0, 0.0], [0.5, 0.5])


def grid(patches, ratios=(2,), cells=(8, 8), block=(8, 8)):
    levels = [[CellBox(lo, hi) for lv, lo, hi in patches if lv == l + 1] for l in range(max([0] + [p[0] for p in patches]))]
    return AmrGrid.from_patches(base(cells, block), list(ratios), levels)


@pytest.mark.parametrize("patches, ratios", [
    ([(1, (4, 4), (8, 8)), (1, (6, 6), (10, 10))], [2]),   # overlap
    ([(1, (3, 4), (8, 8))], [2]),                          # not aligned to the ratio
    ([(1, (12, 12), (18, 18))], [2]),                      # outside the level's domain
    ([(1, (4, 4), (4, 8))], [2]),                          # empty
    ([(1, (4, 4), (8, 8))], [1]),                          # ratio below 2
])
def test_reference_error_paths(patches, ratios):
    with pytest.raises(L.GridError):
        grid(patches, ratios)


def test_more_levels_than_ratios():
    with pytest.raises(L.GridError):
        AmrGrid.from_patches(base(), [2], [[CellBox((4, 4), (8, 8))], [CellBox((8, 8), (12, 12))]])


def test_valid_hierarchies_pass():
    grid([])
    grid([(1, (4, 4), (8, 12)), (1, (8, 4), (12, 12))])
    grid([(1, (4, 4), (12, 12)), (2, (10, 10), (18, 18))], ratios=(2, 2))


@pytest.mark.parametrize("seed", range(40))  # about one in five is a valid hierarchy
def test_verdicts_equal_the_oracle(orc, seed):
    rng = np.random.default_rng(100 + seed)
    cells, block, ratios = (16, 16), (8, 8), [2, 2]
    patches = []
    for lv in (1, 2):
        dom = cells[0] * 2 ** lv
        for _ in range(rng.integers(0, 3)):
            lo = [int(rng.integers(-2, dom)) for _ in range(2)]
            ext = [int(rng.integers(1, 10)) for _ in range(2)]
            if rng.random() < 0.7:  # mostly aligned
                lo = [x - x % 2 for x in lo]
                ext = [e + e % 2 for e in ext]
            patches.append((lv, tuple(lo), tuple(l + e for l, e in zip(lo, ext))))
    try:
        orc.AmrSim(list(cells), list(block), 0.5, ratios, patches)
        oracle_ok = True
    except ValueError:
        oracle_ok = False
    try:
        grid(patches, ratios, cells, block)
        ok = True
    except L.GridError:
        ok = False
    assert ok == oracle_ok, patches
