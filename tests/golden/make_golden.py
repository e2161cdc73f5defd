"""Freeze oracle outputs as golden fixtures (run: python tests/golden/make_golden.py).

The reference ships no golden data; these fixtures pin the oracle (itself
pinned to the reference's known-answer tests, tests/test_oracle_pins.py) so
that any later change to the oracle or the CUDA path is caught bit for bit.
Inputs are built from the reference's own test setups.
"""
import hashlib
import json
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))

import oracle_bind as orc  # noqa: E402
from util import centers, with_ghosts  # noqa: E402

H = 0.4


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def heat_case():
    # tests/heat3d.rs:82-113 setup, 50 steps
    h, kappa, n = 0.1, 0.7, 16
    g = orc.Grid([n] * 3, [n // 2] * 3, [0.0] * 3, [h] * 3)
    st = orc.State(g, [1])
    x = centers([n] * 3, [n // 2] * 3, [0.0] * 3, [h] * 3, 0)
    st.set(0, with_ghosts(np.vectorize(math.cos)(math.pi / (n * h) * x), 1))
    dt = 0.5 / 6.0 * h * h / kappa
    st.heat_run(0, kappa, 0.0, dt, 50)
    return {"steps": 50, "dt": dt, "u": digest(st.interior(0)), "u0_sample": float(st.interior(0)[0, 0, 0, 0])}


def modelc_case(noise, steps):
    # tests/model_c.rs:26-60 setup
    g = orc.Grid([64, 64], [32, 32], [0.0, 0.0], [H, H])
    st = orc.State(g, [1, 1])
    st.initialize_grains([(H, H, 10 * H)], 0.7)
    p = orc.modelc_params(noise=noise)
    dt = 0.2 * (H * H) / p.d_thermal
    t = st.modelc_run(p, 0.0, dt, 7, steps, wiener=True)
    phi, u = st.interior(0), st.interior(1)
    return {"noise": noise, "steps": steps, "dt": dt, "t": t, "phi": digest(phi), "u": digest(u),
            "phi_sample": float(phi[0, 5, 5]), "u_sample": float(u[1, 3, 7])}


def oriented_case(steps):
    # tests/model_c.rs:186-391 setups: three grains, each with its own
    # crystal orientation, theta0 by nearest seed; noisy Euler-Maruyama
    g = orc.Grid([64, 64], [32, 32], [0.0, 0.0], [H, H])
    st = orc.State(g, [1, 1, 0])
    grains = [(6.0, 6.0, 2.0, 0.0), (18.0, 9.0, 2.4, math.pi / 4), (10.0, 20.0, 1.6, 0.3)]
    st.initialize_grains([gr[:3] for gr in grains], 0.7)
    st.initialize_orientations(2, grains)
    p = orc.modelc_params(eps4=0.06, lam=3.19, noise=0.02)
    dt = 0.2 * (H * H) / p.d_thermal
    t = st.modelc_run_oriented(p, 2, 0.0, dt, 11, steps, True)
    phi, u = st.interior(0), st.interior(1)
    return {"steps": steps, "dt": dt, "t": t, "phi": digest(phi), "u": digest(u), "theta0": digest(st.interior(2)),
            "phi_sample": float(phi[1, 9, 20])}


def heat_rk4_case():
    # the heat3d setup above, RungeKutta4 (rk4.rs:40-79) at the same dt
    h, kappa, n = 0.1, 0.7, 16
    g = orc.Grid([n] * 3, [n // 2] * 3, [0.0] * 3, [h] * 3)
    st = orc.State(g, [1])
    x = centers([n] * 3, [n // 2] * 3, [0.0] * 3, [h] * 3, 0)
    st.set(0, with_ghosts(np.vectorize(math.cos)(math.pi / (n * h) * x), 1))
    dt = 0.5 / 6.0 * h * h / kappa
    st.heat_run_rk4(0, kappa, 0.0, dt, 50)
    return {"steps": 50, "dt": dt, "u": digest(st.interior(0))}


def modelc_rk4_oriented_case(steps):
    # tests/model_c.rs:289-336 setup: RungeKutta4 on a rotated grain
    g = orc.Grid([64, 64], [32, 32], [0.0, 0.0], [H, H])
    st = orc.State(g, [1, 1, 0])
    st.initialize_grains([(H, H, 10 * H)], 0.7)
    st.initialize_orientations(2, [(H, H, 10 * H, 0.5)])
    p = orc.modelc_params(eps4=0.06, lam=3.19)
    dt = 0.2 * (H * H) / p.d_thermal
    t = st.modelc_run_rk4(p, 0.0, dt, steps, theta_field=2)
    return {"steps": steps, "dt": dt, "t": t, "phi": digest(st.interior(0)), "u": digest(st.interior(1))}


def main():
    keys = [0, 1, 7, 2**63, 2**64 - 1, orc.mix_key(42, [7, 3, 1, 999])]
    fixtures = {
        "splitmix64": {str(k): orc.splitmix64(k) for k in keys},
        "mix_key": {"42,[7,3,1,999]": orc.mix_key(42, [7, 3, 1, 999]), "1234,[5]": orc.mix_key(1234, [5])},
        "standard_normal": {str(k): float(v) for k, v in zip(keys, orc.standard_normal(np.array(keys, dtype=np.uint64)))},
        "heat3d_16_2x2x2": heat_case(),
        "modelc_64_quiet": modelc_case(0.0, 100),
        "modelc_64_noisy": modelc_case(0.05, 100),
        "modelc_64_oriented_noisy": oriented_case(100),
        "heat3d_16_rk4": heat_rk4_case(),
        "modelc_64_rk4_oriented": modelc_rk4_oriented_case(60),
    }
    (HERE / "oracle_fixtures.json").write_text(json.dumps(fixtures, indent=1, sort_keys=True) + "\n")
    print("wrote", HERE / "oracle_fixtures.json")


if __name__ == "__main__":
    main()
