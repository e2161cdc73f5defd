"""Models of the hot path, mirroring the reference's ``ModelC`` and ``Heat``.

The models here only describe parameters, fields and initial conditions;
their right-hand sides run inside the fused device kernels.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from .core import TIME, wiener
from .rng import fma
from .seeding import Grain, seed_positions  # noqa: F401  (re-exported)

#: Karma-Rappel thin-interface constants (src/physics/phasefield.rs:41-44).
A1 = 0.8836
A2 = 0.6267


class ModelC:
    """Karma-Rappel Model C (src/physics/phasefield.rs:55-116).

    ``noise_amplitude != 0`` is the reference's ``ModelC<Wiener<1>>`` (additive
    noise on phi); 0 is ``ModelC<NoNoise>``.  ``d_thermal`` defaults to
    ``A2 * lambda`` and, as in the reference, is a public field that may be
    set independently.
    """

    def __init__(self, eps4: float, lambda_: float, noise_amplitude: float = 0.0):
        self.eps4 = float(eps4)
        self.lambda_ = float(lambda_)
        self.d_thermal = A2 * self.lambda_
        self.noise_amplitude = float(noise_amplitude)
        self.anisotropy_tol = 1e-8
        self.orientations = False
        self.phi = None
        self.u = None
        self.theta = None

    @classmethod
    def classic(cls, noise_amplitude: float = 0.0) -> "ModelC":
        """eps4 = 0.06, lambda = 3.19 (phasefield.rs:91-95)."""
        return cls(0.06, 3.19, noise_amplitude)

    def stochastic_drivers(self):
        return [wiener(0)] if self.noise_amplitude != 0.0 else []

    def register_fields(self, builder) -> None:
        """phi moved by Time and Wiener(0), u by Time, both ghost 1 (phasefield.rs:335-349)."""
        self.phi = builder.register_driven("phi", 1, [TIME, wiener(0)])
        self.u = builder.register("u", 1)
        if self.orientations:
            # the static crystal orientation theta0, read at cell centres only
            # (ghost width 0; phasefield.rs:342-348)
            self.theta = builder.register_static("theta0", 0)

    def stable_dt(self, spacing) -> Optional[float]:
        """0.2 h^2 / D (phasefield.rs:446-449)."""
        h = min(spacing)
        return 0.2 * (h * h) / self.d_thermal

    def params(self, flux_tol: float = 1e-8) -> N.ModelCParams:
        return N.ModelCParams(self.eps4, self.lambda_, self.d_thermal, self.noise_amplitude, self.anisotropy_tol,
                              flux_tol)

    def enthalpy(self, grid, state) -> float:
        """Total enthalpy h^D * sum(u - phi / 2) over the interior cells, from
        FP64 device sums.  du/dt = D lap u + (dphi/dt) / 2 (phasefield.rs:
        353-422), so without noise and with periodic or zero-flux boundaries a
        step changes it only by rounding: the conservation check of a run in
        either precision.  (The reference has no such diagnostic.)"""
        vol = 1.0
        for h in grid.spacing:
            vol *= h
        return vol * (state.field_sum("u") - 0.5 * state.field_sum("phi"))

    # ------------------------------------------------------ initial state
    def with_orientations(self) -> "ModelC":
        """Per-grain crystal orientations (phasefield.rs:118-125): a static
        theta0 field, and every face's anisotropy taken in its cell's crystal
        frame.  Set theta0 with ``initialize_grains`` (nearest-seed Voronoi)
        or upload it and call ``set_orientations``."""
        self.orientations = True
        return self

    def set_orientations(self, state) -> None:
        """Use the theta0 now in ``state`` for the following steps (cos and
        sin theta0 are computed once, on the host, as the reference does)."""
        N.check(N.lib.lg_modelc_set_orientations(state.handle, state._index("theta0")), state.scheduler.handle)

    def initialize(self, grid, state, seed_center, seed_radius: float, u0: float) -> None:
        """Single tanh seed in an undercooled melt (phasefield.rs:180-189)."""
        self.initialize_seeds(grid, state, [(seed_center, seed_radius)], u0)

    def initialize_seeds(self, grid, state, seeds, u0: float) -> None:
        self.initialize_grains(grid, state, [Grain(c, r, 0.0) for c, r in seeds], u0)

    def initialize_grains(self, grid, state, grains: Sequence[Grain], u0: float) -> None:
        """phi = max over seeds of -tanh((r - r0)/sqrt 2), u = -u0 (phasefield.rs:227-314),
        computed on the host exactly as the reference does, then uploaded."""
        if any(g.orientation != 0.0 for g in grains) and not self.orientations:
            raise ValueError("per-grain orientations need ModelC.with_orientations()")
        arr = np.array([[g.center[0], g.center[1], g.radius, g.orientation] for g in grains], dtype=np.float64)
        if state.alloc.dtype != "f64":
            raise ValueError("initialize_grains targets an FP64 state; upload a cast copy for FP32")
        ptr = arr.ctypes.data_as(C.POINTER(C.c_double)) if len(grains) else None
        N.check(N.lib.lg_modelc_initialize_grains(state.handle, ptr, len(grains), float(u0)),
                state.scheduler.handle)
        if self.orientations:  # theta0 by nearest-seed Voronoi (phasefield.rs:286-311)
            N.check(N.lib.lg_modelc_initialize_orientations(state.handle, state._index("theta0"), ptr, len(grains)),
                    state.scheduler.handle)


class Heat:
    """Isotropic heat equation ``du/dt = kappa * lap(u)``, any dimension
    (tests/heat3d.rs:33-80, examples/heat3d.rs:41-85): u has ghost 1."""

    def __init__(self, kappa: float, dt_factor: Optional[float] = None):
        self.kappa = float(kappa)
        self.dt_factor = dt_factor
        self.u = None

    def stochastic_drivers(self):
        return []

    def register_fields(self, builder) -> None:
        self.u = builder.register("u", 1)

    def stable_dt(self, spacing) -> Optional[float]:
        """0.5/(2D) h^2/kappa (tests/heat3d.rs:76-79), or dt_factor * h^2 / kappa."""
        h = min(spacing)
        if self.dt_factor is not None:
            return self.dt_factor * h * h / self.kappa
        return 0.5 / (2.0 * len(spacing)) * h * h / self.kappa

    def initialize_sine_noise(self, state, seed: int = 42, amp: float = 1e-3) -> None:
        """u = sin(2 pi x) sin(2 pi y) sin(2 pi z) + amp (2 unit_open(mix_key(seed, [gx, gy, gz])) - 1)."""
        N.check(N.lib.lg_heat_initialize_sine_noise(state.handle, self.u, int(seed), float(amp)),
                state.scheduler.handle)
