"""legendre_b200: the B200 device path of legendre's block-stepping hot path.

Importing the package loads ``liblegendre_b200.so`` (built in-tree by
``python -m legendre_b200.build``) and fails if it is missing.
"""
from ._native import LegendreError, exported_symbols  # noqa: F401  (loads the library)
from .core import CudaAllocator, CudaScheduler, DeviceState, FieldSpec, Simulation, StateBuilder, TIME, wiener
from .geometry import CartesianGrid, GridError
from .integrators import EulerMaruyama, FiniteDifference, FiniteVolume, ForwardEuler, RungeKutta4
from .physics import A1, A2, Grain, Heat, ModelC, seed_positions
from .ensemble import Ensemble
from .observe import AsyncObserver, ParquetObserver, Snapshot, cell_centers
from .amr import (AmrGrid, AmrSimulation, BergerOliger, CellBox, ClusterParams, GradientTagger, RegridPolicy,
                  Subcycling)

__all__ = [
    "AmrGrid", "AmrSimulation", "BergerOliger", "CellBox", "ClusterParams", "GradientTagger", "RegridPolicy",
    "Subcycling",
    "AsyncObserver", "ParquetObserver", "Snapshot", "cell_centers",
    "A1", "A2", "CartesianGrid", "CudaAllocator", "CudaScheduler", "DeviceState", "Ensemble", "EulerMaruyama",
    "FieldSpec",
    "FiniteDifference", "FiniteVolume", "ForwardEuler", "Grain", "GridError", "Heat", "LegendreError", "ModelC",
    "RungeKutta4", "Simulation", "StateBuilder", "TIME", "seed_positions", "wiener",
]
