"""Golden fixtures (tests/golden/oracle_fixtures.json, made by make_golden.py)."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import golden.make_golden as mg

FIX = json.loads((Path(__file__).resolve().parent / "golden" / "oracle_fixtures.json").read_text())


def test_rng_fixtures(orc):
    from legendre_b200 import rng
    for k, v in FIX["splitmix64"].items():
        assert orc.splitmix64(int(k)) == v and rng.splitmix64(int(k)) == v
    assert orc.mix_key(42, [7, 3, 1, 999]) == FIX["mix_key"]["42,[7,3,1,999]"]
    keys = np.array([int(k) for k in FIX["standard_normal"]], dtype=np.uint64)
    got = orc.standard_normal(keys)
    assert list(got) == [FIX["standard_normal"][k] for k in FIX["standard_normal"]]


def test_oracle_reproduces_frozen_states():
    assert mg.heat_case() == FIX["heat3d_16_2x2x2"]
    assert mg.modelc_case(0.0, 100) == FIX["modelc_64_quiet"]
    assert mg.modelc_case(0.05, 100) == FIX["modelc_64_noisy"]
    assert mg.oriented_case(100) == FIX["modelc_64_oriented_noisy"]
    assert mg.heat_rk4_case() == FIX["heat3d_16_rk4"]
    assert mg.modelc_rk4_oriented_case(60) == FIX["modelc_64_rk4_oriented"]


@pytest.mark.gpu
def test_cuda_path_matches_frozen_states(sched):
    import legendre_b200 as L
    from util import centers, with_ghosts
    # heat
    h, kappa, n = 0.1, 0.7, 16
    grid = L.CartesianGrid([n] * 3, [n // 2] * 3, [0.0] * 3, [h] * 3)
    sim = L.Simulation(grid, L.FiniteDifference(), L.Heat(kappa), L.ForwardEuler(), sched, L.CudaAllocator("f64"))
    x = centers([n] * 3, [n // 2] * 3, [0.0] * 3, [h] * 3, 0)
    sim.state.upload("u", with_ghosts(np.vectorize(math.cos)(math.pi / (n * h) * x), 1))
    f = FIX["heat3d_16_2x2x2"]
    sim.run(f["dt"], f["steps"])
    assert mg.digest(sim.state.interior("u")) == f["u"]
    # Model C without noise: bitwise
    H = 0.4
    grid = L.CartesianGrid([64, 64], [32, 32], [0.0, 0.0], [H, H])
    model = L.ModelC.classic()
    sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(7), sched, L.CudaAllocator("f64"))
    model.initialize(grid, sim.state, (H, H), 10 * H, 0.7)
    f = FIX["modelc_64_quiet"]
    sim.run(f["dt"], f["steps"])
    assert mg.digest(sim.state.interior("phi")) == f["phi"]
    assert mg.digest(sim.state.interior("u")) == f["u"]
    assert sim.time() == f["t"]
