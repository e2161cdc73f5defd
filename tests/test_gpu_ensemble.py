"""Batched Model C ensembles and the adjoint of the fused step (needs a GPU).

* Each instance of an FP64 ensemble follows its own ``Simulation`` bit for
  bit (noise included).
* The adjoint gradients of L = sum (phi_T - target)^2 agree with central
  finite differences of the FP64 forward -- the device's and the CPU
  oracle's -- to 1e-6 relative.  The reference's flux and anisotropy
  tolerance (A = a_bar where |grad phi|^4 <= 1e-8) makes the forward map jump
  where a face changes branch; a face that does so under the +-h
  perturbation spoils the difference quotient, not the adjoint.  So the
  checks run twice: on the continuous form (tolerance 0) with h = 1e-4, and
  on the reference's tolerance with h = 1e-5, small enough that no face of
  these runs changes branch.
* The FP32 ensemble's gradients (FP32 forward and adjoint; parameter
  partials summed in FP32 within a strip unit, in FP64 across units and
  steps) stay close to the FP64 ones.
* The strip form agrees with the tile form also where it hands units out
  from its work list (more units than one wave of resident warps).
"""
import math

import numpy as np
import pytest
import torch

import legendre_b200 as L
import oracle_bind as orc_mod

pytestmark = pytest.mark.gpu

H = 0.4
LAM, D = 3.19, 2.0


def to_blocks(a, block):
    """(ny, nx) -> (num_blocks, block + 2, block + 2) slabs, zero ghosts."""
    ny, nx = a.shape
    nbx, nby = nx // block, ny // block
    out = np.zeros((nbx * nby, block + 2, block + 2))
    for by in range(nby):
        for bx in range(nbx):
            out[bx + by * nbx, 1:-1, 1:-1] = a[by * block:(by + 1) * block, bx * block:(bx + 1) * block]
    return out


def from_blocks(s, n, block):
    nb = n // block
    out = np.empty((n, n))
    for by in range(nb):
        for bx in range(nb):
            out[by * block:(by + 1) * block, bx * block:(bx + 1) * block] = s[bx + by * nb]
    return out


def seeds_field(ninst, n, radius=5.0):
    """A tanh grain per instance, its centre shifted by the instance index."""
    ys, xs = np.meshgrid((np.arange(n) + 0.5) * H, (np.arange(n) + 0.5) * H, indexing="ij")
    out = np.empty((ninst, n, n))
    for i in range(ninst):
        cx, cy = n * H * (0.45 + 0.03 * i), n * H * (0.5 - 0.02 * i)
        r = np.hypot(xs - cx, ys - cy)
        out[i] = np.maximum(-1.0, -np.tanh((r - radius) / math.sqrt(2.0)))
    return out


def make(sched, n, block, eps4, seeds, noise, dtype="f64", lam=LAM, d=D, tol=1e-8):
    grid = L.CartesianGrid([n, n], [block, block], [0.0, 0.0], [H, H])
    model = L.ModelC(0.05, lam, noise)
    model.d_thermal = d
    model.anisotropy_tol = tol
    return L.Ensemble(grid, model, eps4, seeds, sched, dtype=dtype, flux_tol=tol)


def test_instances_follow_their_own_simulations(sched):
    n, block, noise, steps = 64, 32, 0.02, 15
    eps4, seeds, delta = [0.03, 0.05, 0.065], [3, 4, 5], [0.5, 0.55, 0.6]
    ens = make(sched, n, block, eps4, seeds, noise)
    phi0 = seeds_field(3, n)
    u0 = -np.asarray(delta)[:, None, None] * np.ones((3, n, n))
    ens.set("phi", phi0)
    ens.set("u", u0)
    dt = 0.2 * H * H / D
    ens.run(dt, steps, graph=True)
    got_phi, got_u = ens.get("phi"), ens.get("u")
    for i in range(3):
        grid = L.CartesianGrid([n, n], [block, block], [0.0, 0.0], [H, H])
        model = L.ModelC(eps4[i], LAM, noise)
        model.d_thermal = D
        sim = L.Simulation(grid, L.FiniteVolume(), model, L.EulerMaruyama(seeds[i]), sched, L.CudaAllocator("f64"))
        sim.state.upload("phi", to_blocks(phi0[i], block))
        sim.state.upload("u", to_blocks(u0[i], block))
        sim.run(dt, steps)
        assert np.array_equal(from_blocks(sim.state.interior("phi"), n, block), got_phi[i])
        assert np.array_equal(from_blocks(sim.state.interior("u"), n, block), got_u[i])
    assert ens.time() == (pytest.approx(steps * dt), steps)


# ------------------------------------------------------------- gradients --
N_, BLOCK, NOISE, STEPS, CKPT = 32, 16, 0.005, 24, 7
EPS4, SEEDS, DELTA = [0.04, 0.06], [11, 12], [0.55, 0.5]
DT = 0.2 * H * H / D


def _losses(sched, tol, lam=LAM, d=D, eps4=EPS4, delta=DELTA, phi0=None, target=None, dtype="f64"):
    ens = make(sched, N_, BLOCK, eps4, SEEDS, NOISE, dtype=dtype, lam=lam, d=d, tol=tol)
    ens.set("phi", seeds_field(2, N_) if phi0 is None else phi0)
    ens.set("u", -np.asarray(delta)[:, None, None] * np.ones((2, N_, N_)))
    ens.run(DT, STEPS)
    phi = ens.get("phi")
    ens._destroy()
    if target is None:
        return phi
    return ((phi - target) ** 2).sum(axis=(1, 2))


@pytest.fixture(scope="module", params=[0.0, 1e-8], ids=["continuous", "reference-tol"])
def problem(sched, request):
    tol = request.param
    target = _losses(sched, tol, eps4=[e + 0.01 for e in EPS4], delta=[d + 0.03 for d in DELTA])
    ens = make(sched, N_, BLOCK, EPS4, SEEDS, NOISE, tol=tol)
    ens.set("phi", seeds_field(2, N_))
    ens.set("u", -np.asarray(DELTA)[:, None, None] * np.ones((2, N_, N_)))
    g = ens.value_and_grad(DT, STEPS, CKPT, target)
    ens._destroy()
    return tol, target, g


def _central(f, tol):
    h = 1e-4 if tol == 0.0 else 1e-5
    return (f(+h) - f(-h)) / (2.0 * h)


def _close(adj, fd, rel=1e-6):
    adj, fd = np.atleast_1d(adj), np.atleast_1d(fd)
    assert np.all(np.abs(adj - fd) <= rel * np.maximum(np.abs(fd), 1e-3 * np.abs(fd).max())), (adj, fd)


def test_loss_matches_the_forward(sched, problem):
    tol, target, g = problem
    assert np.allclose(g["loss"], _losses(sched, tol, target=target), rtol=1e-14, atol=0)


def test_parameter_gradients_match_finite_differences(sched, problem):
    tol, target, g = problem
    _close(g["lambda"], _central(lambda h: _losses(sched, tol, lam=LAM + h, target=target), tol))
    _close(g["d_thermal"], _central(lambda h: _losses(sched, tol, d=D + h, target=target), tol))
    _close(g["eps4"], _central(lambda h: _losses(sched, tol, eps4=[e + h for e in EPS4], target=target), tol))
    _close(g["delta"], _central(lambda h: _losses(sched, tol, delta=[d + h for d in DELTA], target=target), tol))


@pytest.mark.parametrize("cell", [(16, 9), (0, 0), (31, 5), (12, 31)])
def test_initial_phi_gradient_matches_finite_differences(sched, problem, cell):
    tol, target, g = problem
    y, x = cell
    base = seeds_field(2, N_)

    def f(h):
        p = base.copy()
        p[:, y, x] += h
        return _losses(sched, tol, phi0=p, target=target)

    _close(g["phi0"][:, y, x], _central(f, tol))


def test_gradients_match_oracle_finite_differences(sched, problem):
    # the CPU restatement of the reference's forward, instance 0, central differences in lambda and eps4
    tol, target, g = problem
    og = orc_mod.Grid([N_, N_], [BLOCK, BLOCK], [0.0, 0.0], [H, H])
    phi0 = seeds_field(2, N_)[0]

    def loss(lam=LAM, eps4=EPS4[0]):
        st = orc_mod.State(og, [1, 1])
        st.set(0, to_blocks(phi0, BLOCK))
        st.set(1, to_blocks(np.full((N_, N_), -DELTA[0]), BLOCK))
        st.modelc_run(orc_mod.modelc_params(eps4=eps4, lam=lam, d_thermal=D, noise=NOISE, tol=tol, flux_tol=tol), 0.0,
                      DT, SEEDS[0], STEPS, wiener=True)
        return ((from_blocks(st.interior(0), N_, BLOCK) - target[0]) ** 2).sum()

    _close(g["lambda"][0], _central(lambda h: loss(lam=LAM + h), tol))
    _close(g["eps4"][0], _central(lambda h: loss(eps4=EPS4[0] + h), tol))


def test_fp32_gradients_close_to_fp64(sched, problem):
    tol, target, g64 = problem
    ens = make(sched, N_, BLOCK, EPS4, SEEDS, NOISE, dtype="f32", tol=tol)
    ens.set("phi", seeds_field(2, N_))
    ens.set("u", -np.asarray(DELTA)[:, None, None] * np.ones((2, N_, N_)))
    g32 = ens.value_and_grad(DT, STEPS, CKPT, target)
    ens._destroy()
    for k in ("lambda", "d_thermal", "eps4", "delta"):
        assert np.all(np.abs(g32[k] - g64[k]) <= 2e-3 * np.abs(g64[k]) + 1e-4 * np.abs(g64[k]).max()), k
    rel = np.linalg.norm(g32["phi0"] - g64["phi0"]) / np.linalg.norm(g64["phi0"])
    assert rel < 5e-3


@pytest.mark.parametrize("dtype,rel", [("f64", 1e-10), ("f32", 2e-4)])
@pytest.mark.parametrize("cells,block,ninst", [((32, 32), 16, 2), ((96, 80), 16, 3), ((64, 64), 64, 1)])
def test_strip_and_tile_adjoints_agree(sched, dtype, rel, cells, block, ninst):
    # the two forms of the step adjoint (warp strips, shared-memory tiles):
    # several strips with a ragged last one, several row runs per instance,
    # block edges inside the instance and instance edges on every side
    nx, ny = cells
    grid = L.CartesianGrid([nx, ny], [block, block], [0.0, 0.0], [H, H])
    ys, xs = np.meshgrid((np.arange(ny) + 0.5) * H, (np.arange(nx) + 0.5) * H, indexing="ij")
    phi0 = np.empty((ninst, ny, nx))
    for i in range(ninst):
        r = np.hypot(xs - nx * H * (0.4 + 0.05 * i), ys - ny * H * (0.55 - 0.04 * i))
        phi0[i] = np.maximum(-1.0, -np.tanh((r - 4.0) / math.sqrt(2.0)))
    eps4, seeds = [0.03 + 0.01 * i for i in range(ninst)], [20 + i for i in range(ninst)]
    target = np.tanh(phi0 * 0.8)
    out = {}
    for kernel in ("tile", "strip"):
        model = L.ModelC(0.05, LAM, 0.01)
        model.d_thermal = D
        ens = L.Ensemble(grid, model, eps4, seeds, sched, dtype=dtype)
        ens.set("phi", phi0)
        ens.set("u", -0.5)
        out[kernel] = ens.value_and_grad(DT, 9, 4, target, kernel=kernel)
        ens._destroy()
    a, b = out["tile"], out["strip"]
    assert np.array_equal(a["loss"], b["loss"])
    for k in ("lambda", "d_thermal", "eps4", "delta"):
        assert np.allclose(b[k], a[k], rtol=rel, atol=rel * np.abs(a[k]).max()), k
    for k in ("phi0", "u0"):
        assert np.linalg.norm(b[k] - a[k]) <= rel * np.linalg.norm(a[k]), k


@pytest.mark.parametrize("dtype,rel", [("f64", 1e-10), ("f32", 2e-4)])
def test_strip_work_list_past_the_first_wave(sched, dtype, rel):
    # 96 instances of 128^2 in 16-row strip units: 96 x 5 strips x 8 row runs
    # = 3840 units, more than one wave of resident warps (148 SMs x 16 warps
    # in FP32, x 8 in FP64), so the strip form hands most units out from its
    # work list; it must still agree with the tile form, and its resident
    # tail must give the same bits
    n, block, ninst = 128, 64, 96
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert ninst * 5 * 8 > sms * 16
    grid = L.CartesianGrid([n, n], [block, block], [0.0, 0.0], [H, H])
    ys, xs = np.meshgrid((np.arange(n) + 0.5) * H, (np.arange(n) + 0.5) * H, indexing="ij")
    phi0 = np.empty((ninst, n, n))
    for i in range(ninst):
        r = np.hypot(xs - n * H * (0.3 + 0.1 * (i % 5)), ys - n * H * (0.35 + 0.07 * (i % 4)))
        phi0[i] = np.maximum(-1.0, -np.tanh((r - 3.0 - (i % 3)) / math.sqrt(2.0)))
    eps4, seeds = [0.02 + 0.01 * (i % 4) for i in range(ninst)], [40 + i for i in range(ninst)]
    target = np.tanh(phi0 * 0.8)
    steps, ckpt = 7, 3
    state_bytes = 2 * ninst * (block + 2) ** 2 * (n // block) ** 2 * (8 if dtype == "f64" else 4)  # phi and u
    out = {}
    for kernel, resident in (("tile", 0), ("strip", 0), ("strip", steps)):
        model = L.ModelC(0.05, LAM, 0.01)
        model.d_thermal = D
        ens = L.Ensemble(grid, model, eps4, seeds, sched, dtype=dtype)
        ens.set("phi", phi0)
        ens.set("u", -0.5)
        out[kernel, resident] = ens.value_and_grad(DT, steps, ckpt, target, kernel=kernel,
                                                   resident_bytes=resident * state_bytes)
        ens._destroy()
    a, b, c = out["tile", 0], out["strip", 0], out["strip", steps]
    assert np.array_equal(a["loss"], b["loss"])
    for k in ("lambda", "d_thermal", "eps4", "delta"):
        assert np.allclose(b[k], a[k], rtol=rel, atol=rel * np.abs(a[k]).max()), k
    for k in ("phi0", "u0"):
        assert np.linalg.norm(b[k] - a[k]) <= rel * np.linalg.norm(a[k]), k
    for k in ("loss", "lambda", "d_thermal", "eps4", "delta", "phi0", "u0"):
        assert np.array_equal(c[k], b[k]), k


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_resident_tail_gives_the_same_bits(sched, dtype):
    # keeping the last segments' states instead of recomputing them changes
    # no bit of the loss, the gradients or the final state, whether some or
    # all segments stay
    steps, ckpt = 11, 3  # segments of 3, 3, 3 and 2 steps
    state_bytes = 2 * 2 * (BLOCK + 2) ** 2 * (N_ // BLOCK) ** 2 * (8 if dtype == "f64" else 4)
    out = []
    for states in (0, 2, 5, steps):
        ens = make(sched, N_, BLOCK, EPS4, SEEDS, NOISE, dtype=dtype)
        ens.set("phi", seeds_field(2, N_))
        ens.set("u", -np.asarray(DELTA)[:, None, None] * np.ones((2, N_, N_)))
        g = ens.value_and_grad(DT, steps, ckpt, seeds_field(2, N_) * 0.5, resident_bytes=states * state_bytes)
        g["phi_T"] = ens.get("phi")
        g["time"] = ens.time()
        ens._destroy()
        out.append(g)
    for g in out[1:]:
        for k in ("loss", "lambda", "d_thermal", "eps4", "delta", "phi0", "u0", "phi_T"):
            assert np.array_equal(g[k], out[0][k]), k
        assert g["time"] == out[0]["time"]


# ------------------------------------------------- Simulation backward API --
def _sim(sched, eps4=EPS4[0], lam=LAM, d=D, seed=SEEDS[0], tol=0.0, phi0=None, delta=DELTA[0], dtype="f64"):
    grid = L.CartesianGrid([N_, N_], [BLOCK, BLOCK], [0.0, 0.0], [H, H])
    model = L.ModelC(eps4, lam, NOISE)
    model.d_thermal = d
    model.anisotropy_tol = tol
    sim = L.Simulation(grid, L.FiniteVolume(tol=tol), model, L.EulerMaruyama(seed), sched, L.CudaAllocator(dtype))
    sim.state.upload("phi", to_blocks(seeds_field(1, N_)[0] if phi0 is None else phi0, BLOCK))
    sim.state.upload("u", to_blocks(np.full((N_, N_), -delta), BLOCK))
    return sim


def test_simulation_value_and_grad_equals_the_one_instance_ensemble(sched):
    """Simulation.value_and_grad gives the one-instance ensemble's loss and
    gradients bit for bit, and leaves the state where run() leaves it."""
    target = _losses(sched, 0.0, eps4=[e + 0.01 for e in EPS4], delta=[d + 0.03 for d in DELTA])[0]
    sim = _sim(sched)
    g = sim.value_and_grad(DT, STEPS, CKPT, target)
    ens = make(sched, N_, BLOCK, EPS4[:1], SEEDS[:1], NOISE, tol=0.0)
    ens.set("phi", seeds_field(1, N_))
    ens.set("u", np.full((1, N_, N_), -DELTA[0]))
    ge = ens.value_and_grad(DT, STEPS, CKPT, target)
    ens._destroy()
    assert g["loss"] == ge["loss"][0]
    for k in ("lambda", "d_thermal", "eps4", "delta"):
        assert g[k] == ge[k][0], k
    assert np.array_equal(g["phi0"], ge["phi0"][0]) and np.array_equal(g["u0"], ge["u0"][0])
    fwd = _sim(sched)
    fwd.run(DT, STEPS)
    assert np.array_equal(sim.state.interior("phi"), fwd.state.interior("phi"))
    assert np.array_equal(sim.state.interior("u"), fwd.state.interior("u"))
    assert sim.time() == fwd.time() and sim.step_index() == fwd.step_index() == STEPS


def test_simulation_value_and_grad_matches_finite_differences(sched):
    """dL/dlambda and dL/dphi_0 of one Simulation against central differences
    of its own forward runs (continuous form, h = 1e-4), to 1e-6."""
    target = _losses(sched, 0.0, eps4=[e + 0.01 for e in EPS4], delta=[d + 0.03 for d in DELTA])[0]
    g = _sim(sched).value_and_grad(DT, STEPS, CKPT, target)

    def loss(**kw):
        s = _sim(sched, **kw)
        s.run(DT, STEPS)
        return ((from_blocks(s.state.interior("phi"), N_, BLOCK) - target) ** 2).sum()

    h = 1e-4
    _close(g["lambda"], (loss(lam=LAM + h) - loss(lam=LAM - h)) / (2 * h))
    _close(g["delta"], (loss(delta=DELTA[0] + h) - loss(delta=DELTA[0] - h)) / (2 * h))
    base = seeds_field(1, N_)[0]
    y, x = 16, 9
    pp, pm = base.copy(), base.copy()
    pp[y, x] += h
    pm[y, x] -= h
    _close(g["phi0"][y, x], (loss(phi0=pp) - loss(phi0=pm)) / (2 * h))
