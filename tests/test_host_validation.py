"""Argument checks of the Python host layer that run before any device call
(CPU): configurations the device paths do not serve are refused with the
error the reference's types would give at compile or construction time."""
import pytest

import legendre_b200 as L
from legendre_b200.amr import AmrGrid, AmrSimulation, Subcycling


def grid2(periodic=(False, False), cells=(64, 64), block=(32, 32)):
    return L.CartesianGrid(list(cells), list(block), [0.0, 0.0], [0.4, 0.4]).with_periodic(list(periodic))


def test_allocator_dtypes():
    assert L.CudaAllocator("f64").code == 0 and L.CudaAllocator("f32").code == 1
    with pytest.raises(ValueError):
        L.CudaAllocator("f16")


@pytest.mark.parametrize("kw, grid", [
    (dict(eps4=[0.05], seeds=[1]), grid2(periodic=(True, False))),   # instances mirror at their edges
    (dict(eps4=[0.05, 0.06], seeds=[1]), grid2()),                    # one seed per instance
    (dict(eps4=[], seeds=[]), grid2()),                               # at least one instance
    (dict(eps4=[0.05], seeds=[1], dtype="f16"), grid2()),
])
def test_ensemble_refuses_what_it_cannot_batch(kw, grid):
    with pytest.raises(ValueError):
        L.Ensemble(grid, L.ModelC(0.05, 3.19), scheduler=None, **kw)


def test_ensemble_refuses_a_3d_grid():
    g = L.CartesianGrid([8, 8, 8], [4, 4, 4], [0.0] * 3, [0.4] * 3)
    with pytest.raises(ValueError):
        L.Ensemble(g, L.ModelC(0.05, 3.19), [0.05], [1], scheduler=None)


def amr_grid():
    return AmrGrid.from_patches(grid2(), [2])


@pytest.mark.parametrize("args, exc", [
    ((L.FiniteVolume(), L.ModelC(0.05, 3.19), Subcycling(1), L.CudaAllocator("f32")), ValueError),  # FP64 only
    ((L.FiniteDifference(), L.ModelC(0.05, 3.19), Subcycling(1), L.CudaAllocator("f64")), TypeError),
    ((L.FiniteVolume(), object(), Subcycling(1), L.CudaAllocator("f64")), TypeError),
    ((L.FiniteVolume(), L.ModelC(0.05, 3.19), L.RungeKutta4(), L.CudaAllocator("f64")), TypeError),
])
def test_amr_simulation_refuses_unserved_configurations(args, exc):
    disc, model, integ, alloc = args
    with pytest.raises(exc):
        AmrSimulation(amr_grid(), disc, model, integ, None, alloc)


def test_amr_simulation_refuses_a_3d_base():
    g = L.CartesianGrid([8, 8, 8], [4, 4, 4], [0.0] * 3, [0.4] * 3)
    with pytest.raises(ValueError):
        AmrSimulation(AmrGrid.from_patches(g, [2]), L.FiniteVolume(), L.ModelC(0.05, 3.19), Subcycling(1), None,
                      L.CudaAllocator("f64"))
