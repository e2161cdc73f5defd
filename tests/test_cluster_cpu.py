"""The library's Berger-Rigoutsos clustering (lg_amr_cluster, the host code
its regrids run) against the oracle's restatement and the reference's own
cluster tests (amr/cluster.rs:320-431), on the CPU."""
import numpy as np
import pytest

from legendre_b200 import LegendreError
from legendre_b200.amr import ClusterParams, cluster


def art(rows):
    return [(c, r) for r, row in enumerate(rows) for c, ch in enumerate(row) if ch == "x"]


def boxes_of(flags, eff, mw):
    return [(b.lo, b.hi) for b in cluster(flags, ClusterParams(eff, mw))]


CASES = [
    (art(["xxxx", "xxxx", "xxxx"]), 0.8, 4),                                          # cluster.rs:320-331
    (art(["xx....xxx", "xx....xxx", "......xxx"]), 0.8, 4),                           # cluster.rs:333-346
    (art(["xx......"] * 4 + ["xxxxxxxx"] * 2), 0.95, 2),                              # cluster.rs:348-374
    (art(["x.....x", "x.....x", ".x...x.", ".x...x.", "..x.x..", "..xxx.."]), 0.7, 1),  # cluster.rs:376-395
    ([(i, i) for i in range(8)], 0.8, 1),                                             # cluster.rs:397-431
    ([(i, i) for i in range(8)], 0.8, 2),
]


@pytest.mark.parametrize("flags, eff, mw", CASES)
def test_reference_cases_equal_the_oracle(orc, flags, eff, mw):
    assert boxes_of(flags, eff, mw) == orc.cluster(sorted(flags), eff, mw)


def test_dense_rectangle_is_one_box():
    assert boxes_of(art(["xxxx", "xxxx", "xxxx"]), 0.8, 4) == [((0, 0), (4, 3))]


@pytest.mark.parametrize("seed", range(12))
def test_random_flag_sets_equal_the_oracle_in_any_order(orc, seed):
    rng = np.random.default_rng(seed)
    # blobs of flags on a 96 x 80 level, as a gradient tagger leaves them
    n = rng.integers(1, 5)
    cells = set()
    for _ in range(n):
        cx, cy, r = rng.integers(0, 96), rng.integers(0, 80), rng.integers(2, 14)
        for x in range(max(0, cx - r), min(96, cx + r)):
            for y in range(max(0, cy - r), min(80, cy + r)):
                if (x - cx) ** 2 + (y - cy) ** 2 <= r * r and rng.random() < 0.9:
                    cells.add((x, y))
    flags = sorted(cells)
    eff, mw = [(0.8, 4), (0.7, 2), (0.9, 1)][seed % 3]
    want = orc.cluster(flags, eff, mw)
    assert boxes_of(flags, eff, mw) == want
    shuffled = [flags[i] for i in rng.permutation(len(flags))]
    assert boxes_of(shuffled, eff, mw) == want


def test_no_flags_no_boxes():
    assert cluster([], ClusterParams()) == []


@pytest.mark.parametrize("eff, mw", [(0.0, 4), (1.5, 4), (0.8, 0)])
def test_invalid_parameters_are_refused(eff, mw):
    with pytest.raises(LegendreError):
        cluster([(0, 0)], ClusterParams(eff, mw))


# ---- the reference's own assertions (amr/cluster.rs:306-431), checked on the
# product's clustering directly, not through the oracle
def _cover_disjoint(flags, boxes):
    """cluster.rs:306-319: every flag in exactly one box; boxes pairwise
    disjoint (half-open)."""
    for f in flags:
        n = sum(1 for b in boxes if b[0][0] <= f[0] < b[1][0] and b[0][1] <= f[1] < b[1][1])
        assert n == 1, f"flag {f} covered by {n} boxes: {boxes}"
    for i, a in enumerate(boxes):
        for b in boxes[i + 1:]:
            overlap = all(max(a[0][d], b[0][d]) < min(a[1][d], b[1][d]) for d in range(2))
            assert not overlap, f"boxes overlap: {a} {b}"


def _cells(b):
    return (b[1][0] - b[0][0]) * (b[1][1] - b[0][1])


def _flags_in(flags, b):
    return sum(1 for f in flags if b[0][0] <= f[0] < b[1][0] and b[0][1] <= f[1] < b[1][1])


def test_reference_dense_rectangle_is_one_full_box():
    # cluster.rs:320-331
    flags = art(["xxxx", "xxxx", "xxxx"])
    boxes = boxes_of(flags, 0.8, 4)
    assert boxes == [((0, 0), (4, 3))]
    _cover_disjoint(flags, boxes)


def test_reference_islands_split_at_holes():
    # cluster.rs:333-346: two islands, each boxed tightly
    flags = art(["xx....xxx", "xx....xxx", "......xxx"])
    boxes = boxes_of(flags, 0.8, 4)
    assert len(boxes) == 2, boxes
    _cover_disjoint(flags, boxes)
    assert sum(_cells(b) for b in boxes) == len(flags)


def test_reference_l_shape_splits_at_inflection():
    # cluster.rs:348-374: two boxes cover the L exactly
    flags = art(["xx......"] * 4 + ["xxxxxxxx"] * 2)
    boxes = boxes_of(flags, 0.95, 2)
    _cover_disjoint(flags, boxes)
    assert sum(_cells(b) for b in boxes) == len(flags), boxes
    assert len(boxes) == 2, boxes


def test_reference_v_shape_is_covered_efficiently():
    # cluster.rs:376-395
    flags = art(["x.....x", "x.....x", ".x...x.", ".x...x.", "..x.x..", "..xxx.."])
    boxes = boxes_of(flags, 0.7, 1)
    _cover_disjoint(flags, boxes)
    assert len(flags) / sum(_cells(b) for b in boxes) >= 0.7, boxes


def test_reference_diagonal_stripe_bisects_past_the_anomaly():
    # cluster.rs:397-431: bisection makes progress on a 45-degree stripe;
    # with a width floor every box keeps at least half its cells flagged
    flags = [(i, i) for i in range(8)]
    boxes = boxes_of(flags, 0.8, 1)
    _cover_disjoint(flags, boxes)
    assert len(flags) / sum(_cells(b) for b in boxes) >= 0.8, boxes
    boxes = boxes_of(flags, 0.8, 2)
    _cover_disjoint(flags, boxes)
    for b in boxes:
        assert _flags_in(flags, b) / _cells(b) >= 0.5, (b, boxes)
