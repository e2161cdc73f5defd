"""The oracle's RungeKutta4 (rk4.rs:40-79) against the reference's pins:

* heat decays as the discrete eigenmode times the RK4 amplification factor
  1 - z + z^2/2 - z^3/6 + z^4/24 per step (tests/heat.rs:86-168, 1e-10);
* multi-grain Model C stepped by RK4 carries theta0 through the stage states
  and stays bounded (tests/model_c.rs:289-336);
* the result does not depend on the thread count (tests/heat.rs:178-183).
"""
import math

import numpy as np

import oracle_bind as orc
from util import centers, relative_eq


def test_rk4_heat_matches_discrete_eigenmode_decay():
    n, h, kappa, steps = 32, 0.1, 0.7, 200
    cells, block = [n, n], [n // 4, n // 4]
    g = orc.Grid(cells, block, [0.0, 0.0], [h, h])
    st = orc.State(g, [1])
    kx = math.pi / (n * h)
    x = centers(cells, block, [0.0, 0.0], [h, h], 0)
    u0 = np.zeros((g.num_blocks(),) + g.slab_shape(1))
    u0[:, 1:-1, 1:-1] = np.cos(kx * x)
    st.set(0, u0)
    dt = 0.25 * h * h / kappa
    st.heat_run_rk4(0, kappa, 0.0, dt, steps, threads=4)
    lam = (2.0 - 2.0 * math.cos(kx * h)) / (h * h)
    z = dt * kappa * lam
    factor = (1.0 - z + z * z / 2.0 - z * z * z / 6.0 + z * z * z * z / 24.0) ** steps
    assert np.all(relative_eq(st.interior(0), factor * np.cos(kx * x), 1e-10, 1e-12))


def test_rk4_stage_states_carry_the_orientation_field():
    n, H = 64, 0.4
    g = orc.Grid([n, n], [n // 2, n // 2], [0.0, 0.0], [H, H])
    st = orc.State(g, [1, 1, 0])
    st.initialize_grains([(H, H, 10 * H)], 0.7)
    st.initialize_orientations(2, [(H, H, 10 * H, 0.5)])
    p = orc.modelc_params(eps4=0.06, lam=3.19)
    st.modelc_run_rk4(p, 0.0, 0.2 * H * H / p.d_thermal, 200, theta_field=2, threads=4)
    phi = st.interior(0)
    assert np.all(np.isfinite(phi)) and np.all(np.abs(phi) < 1.2)
    assert np.all(st.interior(2) == 0.5)


def test_rk4_is_thread_count_independent():
    # tests/heat.rs:178-183 (rk4_parallel_is_bitwise_identical_to_serial),
    # and the multi-grain Model C form
    n, h, kappa = 32, 0.1, 0.7
    cells, block = [n, n], [n // 4, n // 4]
    g = orc.Grid(cells, block, [0.0, 0.0], [h, h])
    x = centers(cells, block, [0.0, 0.0], [h, h], 0)
    out = []
    for threads in (1, 4):
        st = orc.State(g, [1])
        u0 = np.zeros((g.num_blocks(),) + g.slab_shape(1))
        u0[:, 1:-1, 1:-1] = np.cos(math.pi / (n * h) * x)
        st.set(0, u0)
        st.heat_run_rk4(0, kappa, 0.0, 0.25 * h * h / kappa, 50, threads=threads)
        out.append(st.interior(0))
    assert np.array_equal(out[0], out[1])
    H = 0.4
    g = orc.Grid([64, 64], [16, 16], [0.0, 0.0], [H, H])
    res = []
    for threads in (1, 4):
        st = orc.State(g, [1, 1, 0])
        st.initialize_grains([(8.0, 8.0, 3.0), (17.0, 15.0, 2.0)], 0.7)
        st.initialize_orientations(2, [(8.0, 8.0, 3.0, 0.2), (17.0, 15.0, 2.0, 1.1)])
        p = orc.modelc_params(eps4=0.06, lam=3.19)
        st.modelc_run_rk4(p, 0.0, 0.2 * H * H / p.d_thermal, 40, theta_field=2, threads=threads)
        res.append((st.interior(0), st.interior(1)))
    assert all(np.array_equal(a, b) for a, b in zip(res[0], res[1]))
