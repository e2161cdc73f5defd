"""legendre_b200: the B200 device path of legendre's block-stepping hot path.

The public names below load ``liblegendre_b200.so`` (built in-tree by
``python legendre_b200/build.py``) on first use and fail loudly if it is
missing: there is no CPU fallback.  The pure-Python modules ``rng`` and
``seeding`` (the counter generator and the example's grain placement) load
nothing, so a CPU-only caller can use them without mapping the library.
"""
from __future__ import annotations

import importlib

_EXPORTS = {
    "_native": ("LegendreError", "exported_symbols"),
    "core": ("CudaAllocator", "CudaScheduler", "DeviceState", "FieldSpec", "Simulation", "StateBuilder", "TIME",
             "wiener"),
    "geometry": ("CartesianGrid", "GridError"),
    "integrators": ("EulerMaruyama", "FiniteDifference", "FiniteVolume", "ForwardEuler", "RungeKutta4"),
    "physics": ("A1", "A2", "Heat", "ModelC"),
    "seeding": ("Grain", "seed_positions"),
    "ensemble": ("Ensemble",),
    "observe": ("AsyncObserver", "ParquetObserver", "Snapshot", "cell_centers"),
    "amr": ("AmrGrid", "AmrSimulation", "BergerOliger", "CellBox", "ClusterParams", "GradientTagger",
            "RegridPolicy", "Subcycling"),
}
_OWNER = {name: mod for mod, names in _EXPORTS.items() for name in names}
_SUBMODULES = set(_EXPORTS) | {"rng", "build"}

__all__ = sorted(_OWNER)


def __getattr__(name: str):
    if name in _OWNER:
        value = getattr(importlib.import_module("." + _OWNER[name], __name__), name)
    elif name in _SUBMODULES:
        value = importlib.import_module("." + name, __name__)
    else:
        raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
    globals()[name] = value
    return value


def __dir__():
    return sorted(set(globals()) | set(_OWNER) | _SUBMODULES)
