"""bench.py's reference arm on the host: rank 0 times the oracle (the C++
restatement of the reference's CPU path) and prints one JSON line with the
GPU arm's metric, unit and direction, the CPU sample it timed and a zero-copy
e2e block.  Small grids stand in for the configurations' full sizes."""
import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


class _Args:
    steps, warmup, gpus = 2, 3, 1


def _line(capsys, cfg):
    sys.path.insert(0, str(ROOT))
    import bench

    bench.run_reference(_Args(), cfg)
    out = capsys.readouterr().out.strip().splitlines()
    assert len(out) == 1
    return json.loads(out[0])


@pytest.mark.parametrize("name, over", [
    ("c2", dict(cells=128, block=32)),
    ("c3o", dict(cells=126, block=63, grains=6)),
])
def test_reference_arm_line(capsys, monkeypatch, name, over):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "0")
    cfg = dict(bench.CONFIGS[name], **over)
    d = _line(capsys, cfg)
    assert d["impl"] == "reference"
    assert (d["metric"], d["unit"], d["higher_is_better"]) == ("Gcell-updates/s", "Gcell-updates/s", True)
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["config"]["workload"] == cfg["workload"] and d["config"]["cells"] == cfg["cells"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["sample"].startswith("2 of 2 steps")
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_roofline_object_carries_both_denominators_and_the_captured_figures():
    import types

    sys.path.insert(0, str(ROOT))
    import bench

    a = types.SimpleNamespace(cells=None, noise=None, integrator="em", variant=0, config="c2", dtype="f64")
    r = bench.hbm_roofline(1600.0, 6400.0, "measured", traffic=bench.traffic(a, 4096 ** 2),
                           algorithmic_bytes_per_cell=32)
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert r["frac"] == 0.25 and r["frac_nominal"] == 1600.0 / 8000.0 and r["peak_kind"] == "measured"
    assert r["traffic"] == bench.TRAFFIC_PER_CELL[("c2", "f64")] * 4096 ** 2
    assert bench.NCU_PIPES[("c2", "f64")]["fp64_pipe"] > 0
    # the ncu figures belong to the captured configuration only
    for over in (dict(cells=512), dict(noise=0.0), dict(integrator="rk4"), dict(variant=3)):
        b = types.SimpleNamespace(**dict(vars(a), **over))
        assert not bench.captured(b) and bench.traffic(b, 4096 ** 2) is None


def test_tip_extents_find_each_grains_four_tips():
    import numpy as np

    sys.path.insert(0, str(ROOT))
    import bench

    n, h = 96, 0.4
    x = (np.arange(n) + 0.5) * h
    X, Y = np.meshgrid(x, x)  # rows = y
    grains = [((10.2, 11.0), 3.1), ((26.0, 24.4), 4.4)]

    def field(scale):
        phi = np.full((n, n), -1.0)
        for (cx, cy), r in grains:
            phi = np.maximum(phi, np.tanh((scale * r - np.hypot(X - cx, Y - cy)) / (2 * h)))
        return phi

    for scale in (1.0, 1.25):
        ext = bench.tip_extents(field(scale), [c for c, _ in grains], h)
        for g, (_, r) in enumerate(grains):
            assert np.all(np.abs(ext[g] - scale * r) < 0.02 * h)
    # +x agrees with the single-tip helper
    phi = field(1.0)
    (cx, cy), _ = grains[1]
    assert abs(bench.tip_extents(phi, [(cx, cy)], h)[0, 0] + cx - bench.tip_position(phi, int(cy / h), cx, h)) < 1e-12
    # a centre outside the solid has no tips
    assert np.all(np.isnan(bench.tip_extents(phi, [(1.0, 1.0)], h)))
