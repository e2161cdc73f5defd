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
    assert d["ms_per_step"] > 0
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

    a = types.SimpleNamespace(cells=None, noise=None, integrator="em", variant=0, config="c3", dtype="f64")
    r = bench.hbm_roofline(1600.0, 6400.0, "measured", traffic=bench.traffic(a, 10080 ** 2),
                           algorithmic_bytes_per_cell=32)
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert r["frac"] == 0.25 and r["frac_nominal"] == 1600.0 / 8000.0 and r["peak_kind"] == "measured"
    assert r["traffic"] == bench.TRAFFIC_PER_CELL[("c3", "f64")] * 10080 ** 2
    # the captured traffic is close to the algorithmic 32 B per cell
    assert 28.0 < bench.TRAFFIC_PER_CELL[("c3", "f64")] < 36.0
    assert bench.NCU_INST[("c3", "f64")]["fp64_inst_per_cell"] > 0
    assert bench.ncu_capture_config(types.SimpleNamespace(**dict(vars(a), variant=bench.CAPTURED_VARIANT)))
    # the ncu figures belong to the captured configuration only
    for over in (dict(cells=512), dict(noise=0.0), dict(integrator="rk4"), dict(variant=3)):
        b = types.SimpleNamespace(**dict(vars(a), **over))
        assert not bench.ncu_capture_config(b) and bench.traffic(b, 10080 ** 2) is None


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


def _fake_clock():
    return {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 10}


@pytest.mark.parametrize("config", ["c2", "c3", "c3o"])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("observe", [0, 5])
def test_model_c_line_assembles_for_every_uniform_config(config, dtype, observe):
    """The line of every uniform Model C configuration assembles from fake
    timings, with and without the observer block, and is valid JSON with the
    contract's keys."""
    sys.path.insert(0, str(ROOT))
    import bench

    argv = ["--config", config, "--dtype", dtype, "--steps", "20", "--warmup", "5"]
    if observe:
        argv += ["--observe-every", str(observe)]
    args, cfg = bench.parse_args(argv)
    cells = cfg["cells"] ** 2
    ms = 40.0
    observed = bench.observer_block(args, 1, cells, ms, 41.0, 4, 0) if observe else None
    e2e = {"value": 1.0, "unit": "Gcell-updates/s", "h2d_bytes_per_step": 8.0, "d2h_bytes_per_step": 8.0}
    cpu = {"value": 0.1, "unit": "Gcell-updates/s", "cores": 16, "kind": "port", "sample": "x"}
    line = bench.model_c_line(args, cfg, 1, ms, _fake_clock(), 20, 3, e2e, observed, None, cpu, 6538.6, "measured")
    d = json.loads(json.dumps(line))
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e",
              "gpu_launches", "clocks"):
        assert k in d, k
    assert d["steps"] == 20 and d["warmup"] == 5 and d["dtype"] == dtype
    assert abs(d["ms_per_step"] * d["steps"] - ms) < 1e-9
    assert abs(d["value"] - cells * 20 / (ms / 1e3) / 1e9) < 1e-9
    assert d["config"]["workload"] == cfg["workload"]
    r = d["roofline"]
    esz = 8 if dtype == "f64" else 4
    bpc = 4 * esz + (2 * esz if config == "c3o" else 0)
    assert r["algorithmic_bytes_per_cell"] == bpc
    assert abs(r["achieved"] - bpc * cells / (ms / 20 / 1e3) / 1e9) < 1e-6
    assert abs(r["frac"] - r["achieved"] / 6538.6) < 1e-12
    if observe:
        assert d["observer"]["captured"] == 4 and d["observer"]["every"] == observe


def test_default_config_is_the_full_scale_grid():
    sys.path.insert(0, str(ROOT))
    import bench

    args, cfg = bench.parse_args([])
    assert args.config == "c3" and cfg["cells"] == 10080 and cfg["block"] == 126 and args.dtype == "f64"


def test_no_function_local_shadows_a_module_level_name():
    """A local assigned anywhere in a function hides the module-level name of
    the same spelling for the whole function (the class of bug that made
    main() raise UnboundLocalError): no function of bench.py may assign a
    name that the module defines as a function or class."""
    import symtable

    src = (ROOT / "bench.py").read_text()
    top = symtable.symtable(src, "bench.py", "exec")
    module_defs = {s.get_name() for s in top.get_symbols() if s.is_namespace()}

    def walk(tab, path):
        for sym in tab.get_symbols():
            if tab.get_type() == "function" and sym.is_assigned() and sym.get_name() in module_defs \
                    and not sym.is_global():
                if not sym.is_namespace():
                    raise AssertionError(f"{path}: local {sym.get_name()!r} shadows a module-level definition")
        for child in tab.get_children():
            walk(child, f"{path}.{child.get_name()}")

    walk(top, "bench")


def test_reference_arm_maps_no_product_library(tmp_path):
    """The reference arm loads the oracle's library only: its process never
    maps liblegendre_b200.so."""
    import subprocess

    code = (
        "import json, os, sys\n"
        f"sys.path.insert(0, {str(ROOT)!r})\n"
        "os.environ['RANK'] = '0'\n"
        "import bench\n"
        "class A: steps, warmup, gpus = 1, 1, 1\n"
        "cfg = dict(bench.CONFIGS['c2'], cells=64, block=32)\n"
        "bench.run_reference(A(), cfg)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('PRODUCT_MAPPED' if 'liblegendre_b200' in maps else 'PRODUCT_NOT_MAPPED')\n"
        "print('ORACLE_MAPPED' if 'liblegendre_oracle' in maps else 'ORACLE_NOT_MAPPED')\n"
    )
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "PRODUCT_NOT_MAPPED" in out.stdout and "ORACLE_MAPPED" in out.stdout
    line = json.loads(out.stdout.strip().splitlines()[0])
    assert line["impl"] == "reference" and line["ms_per_step"] > 0


def test_compute_roofline_fractions():
    sys.path.insert(0, str(ROOT))
    import bench

    peaks = {"dfma_per_s": 20e12, "ffma_per_s": 70e12, "imad_per_s": 35e12, "alu_per_s": 35e12, "sms": 148,
             "clock_mhz": 1965.0}
    ncu = {"capture": "x", "inst_per_cell": 464.0, "fp64_inst_per_cell": 266.0}
    r = bench.compute_roofline(peaks, 1965.0, 50e9, ncu)
    ceiling = 148 * 4 * 32 * 1965e6
    assert abs(r["issue_ceiling_thread_inst_per_s"] - ceiling) < 1.0
    assert abs(r["issue_frac"] - 464.0 * 50e9 / ceiling) < 1e-12
    assert abs(r["fp64_frac"] - 266.0 * 50e9 / 20e12) < 1e-12
    assert bench.compute_roofline(peaks, None, 50e9, None)["issue_frac"] is None
    assert bench.compute_roofline(None, 1965.0, 50e9, ncu) is None
