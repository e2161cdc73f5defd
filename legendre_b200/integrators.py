"""Integrators and discretisation policies of the device path.

``ForwardEuler`` and ``EulerMaruyama`` mirror src/integrators/euler.rs and
euler_maruyama.rs; their ``run`` dispatches the fused device step for the
model at hand.  ``FiniteVolume`` / ``FiniteDifference`` are the reference's
discretisation policies (finite_volume.rs:41-50, finite_difference.rs:23-43).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _native as N
from .physics import Heat, ModelC


@dataclass
class FiniteVolume:
    tol: float = 1e-8


@dataclass
class FiniteDifference:
    pass


def _flags(graph: bool) -> int:
    return N.LG_RUN_GRAPH if graph else 0


@dataclass
class ForwardEuler:
    """Explicit Euler, deterministic models only (euler.rs:13-55)."""

    def suggested_dt(self, model, grid):
        return model.stable_dt(grid.spacing)

    def validate(self, model, grid, disc):
        if model.stochastic_drivers():
            raise TypeError("ForwardEuler integrates deterministic models only; use EulerMaruyama")
        _validate_model(model, grid, disc)

    def run(self, sim, dt, nsteps, graph=False, variant=0):
        _run(sim, dt, nsteps, seed=0, graph=graph, variant=variant)


@dataclass
class EulerMaruyama:
    """Euler-Maruyama (euler_maruyama.rs:21-75); ``seed`` keys the noise."""

    seed: int = 0

    def suggested_dt(self, model, grid):
        return model.stable_dt(grid.spacing)

    def validate(self, model, grid, disc):
        _validate_model(model, grid, disc)

    def run(self, sim, dt, nsteps, graph=False, variant=0):
        _run(sim, dt, nsteps, seed=self.seed, graph=graph, variant=variant)


@dataclass
class RungeKutta4:
    """Classic fourth-order Runge-Kutta (rk4.rs:13-79), deterministic models
    only (the reference enforces NoNoise): Model C with no noise, or heat.
    Four fused stage launches per step on the device."""

    def suggested_dt(self, model, grid):
        return model.stable_dt(grid.spacing)

    def validate(self, model, grid, disc):
        if model.stochastic_drivers() or getattr(model, "noise_amplitude", 0.0) != 0.0:
            raise TypeError("RungeKutta4 integrates deterministic models only; use EulerMaruyama")
        _validate_model(model, grid, disc)

    def run(self, sim, dt, nsteps, graph=False, variant=0):
        st = sim.state
        ctx = sim.scheduler.handle
        if isinstance(sim.model, ModelC):
            p = sim.model.params(flux_tol=sim.disc.tol)
            N.check(N.lib.lg_modelc_rk4_run(st.handle, C.byref(p), dt, nsteps, _flags(graph)), ctx)
        elif isinstance(sim.model, Heat):
            N.check(N.lib.lg_heat_rk4_run(st.handle, sim.model.u, sim.model.kappa, dt, nsteps, _flags(graph)), ctx)
        else:
            raise TypeError(f"no device path for model {type(sim.model).__name__}")


def _validate_model(model, grid, disc):
    if isinstance(model, ModelC):
        if grid.dim != 2:
            raise TypeError("Model C runs on a 2-D grid")
        if not isinstance(disc, FiniteVolume):
            raise TypeError("Model C's anisotropic divergence needs the FiniteVolume policy")
    elif isinstance(model, Heat):
        if not isinstance(disc, (FiniteDifference, FiniteVolume)):
            raise TypeError("the heat model needs a Laplacian discretisation")
    else:
        raise TypeError(f"no device path for model {type(model).__name__}")


def _run(sim, dt, nsteps, seed, graph, variant):
    st = sim.state
    ctx = sim.scheduler.handle
    if isinstance(sim.model, ModelC):
        p = sim.model.params(flux_tol=sim.disc.tol)
        N.check(N.lib.lg_modelc_em_run(st.handle, C.byref(p), dt, int(seed) & ((1 << 64) - 1), nsteps, int(variant),
                                       _flags(graph)), ctx)
    elif isinstance(sim.model, Heat):
        N.check(N.lib.lg_heat_fe_run(st.handle, sim.model.u, sim.model.kappa, dt, nsteps, _flags(graph)), ctx)
    else:
        raise TypeError(f"no device path for model {type(sim.model).__name__}")
