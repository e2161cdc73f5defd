"""ctypes binding of the CPU oracle (oracle/liblegendre_oracle.so) for the tests.

The oracle restates the reference's SerialScheduler path on the CPU; tests use
it only as the checker of the CUDA library.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
_PATH = ROOT / "oracle" / "liblegendre_oracle.so"


class Params(C.Structure):
    _fields_ = [("eps4", C.c_double), ("lambda_", C.c_double), ("d_thermal", C.c_double),
                ("noise_amplitude", C.c_double), ("anisotropy_tol", C.c_double), ("flux_tol", C.c_double)]


def _load():
    if not _PATH.exists():
        import importlib.util
        spec = importlib.util.spec_from_file_location("legendre_b200_build", ROOT / "legendre_b200" / "build.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build_oracle()
    lib = C.CDLL(str(_PATH))
    p, i64, u64, d = C.c_void_p, C.c_int64, C.c_uint64, C.c_double
    pd, pi64 = C.POINTER(C.c_double), C.POINTER(C.c_int64)
    sigs = {
        "orc_splitmix64": (u64, [u64]),
        "orc_mix_key": (u64, [u64, C.POINTER(C.c_uint64), i64]),
        "orc_unit_open": (d, [u64]),
        "orc_standard_normal": (d, [u64]),
        "orc_standard_normal_batch": (None, [C.POINTER(C.c_uint64), i64, pd]),
        "orc_grid_create": (p, [C.c_int, pi64, pi64, pd, pd, C.POINTER(C.c_int)]),
        "orc_grid_destroy": (None, [p]),
        "orc_grid_num_blocks": (i64, [p]),
        "orc_grid_block_len": (i64, [p, C.c_int]),
        "orc_grid_face_neighbor": (i64, [p, i64, C.c_int, C.c_int]),
        "orc_grid_cell_center": (None, [p, i64, pi64, pd]),
        "orc_grid_cell_key": (C.c_int, [p, C.c_int, i64, C.POINTER(C.c_uint64)]),
        "orc_state_create": (p, [p, C.c_int, C.POINTER(C.c_int)]),
        "orc_state_destroy": (None, [p]),
        "orc_state_set_field": (None, [p, C.c_int, pd]),
        "orc_state_get_field": (None, [p, C.c_int, pd]),
        "orc_fill_ghosts_mirror": (None, [p, p, C.c_int]),
        "orc_heat_run": (d, [p, p, C.c_int, d, d, d, i64, C.c_int]),
        "orc_modelc_run": (d, [p, p, C.POINTER(Params), d, d, u64, i64, C.c_int, C.c_int]),
        "orc_modelc_drift": (None, [p, p, C.POINTER(Params), pd, pd]),
        "orc_modelc_initialize_grains": (None, [p, p, pd, i64, d]),
        "orc_modelc_run_oriented": (d, [p, p, C.POINTER(Params), C.c_int, d, d, u64, i64, C.c_int, C.c_int]),
        "orc_modelc_initialize_orientations": (None, [p, p, C.c_int, pd, i64]),
        "orc_heat_run_rk4": (d, [p, p, C.c_int, d, d, d, i64, C.c_int]),
        "orc_modelc_run_rk4": (d, [p, p, C.POINTER(Params), C.c_int, d, d, i64, C.c_int]),
        "orc_num_threads_available": (C.c_int, []),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def splitmix64(z):
    return lib.orc_splitmix64(z)


def mix_key(seed, parts):
    arr = (C.c_uint64 * len(parts))(*parts)
    return lib.orc_mix_key(seed, arr, len(parts))


def standard_normal(keys):
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    out = np.empty(keys.size, dtype=np.float64)
    lib.orc_standard_normal_batch(keys.ctypes.data_as(C.POINTER(C.c_uint64)), keys.size,
                                  out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


class Grid:
    """The oracle's CartesianGrid<D>."""

    def __init__(self, cells, block, origin, spacing, periodic=None):
        D = len(cells)
        periodic = periodic or [False] * D
        self.D, self.cells, self.block = D, tuple(cells), tuple(block)
        self.origin, self.spacing, self.periodic = tuple(origin), tuple(spacing), tuple(periodic)
        self.h = lib.orc_grid_create(D, (C.c_int64 * D)(*cells), (C.c_int64 * D)(*block), (C.c_double * D)(*origin),
                                     (C.c_double * D)(*spacing), (C.c_int * D)(*[int(x) for x in periodic]))
        if not self.h:
            raise ValueError("invalid grid")

    def __del__(self):
        if getattr(self, "h", None):
            lib.orc_grid_destroy(self.h)

    def num_blocks(self):
        return lib.orc_grid_num_blocks(self.h)

    def block_len(self, g):
        return lib.orc_grid_block_len(self.h, g)

    def face_neighbor(self, b, dim, direction):
        r = lib.orc_grid_face_neighbor(self.h, b, dim, direction)
        return None if r < 0 else r

    def cell_center(self, b, idx):
        out = (C.c_double * 3)()
        ii = (C.c_int64 * 3)(*(list(idx) + [0] * (3 - len(idx))))
        lib.orc_grid_cell_center(self.h, b, ii, out)
        return tuple(out[: self.D])

    def slab_shape(self, g):
        return tuple(b + 2 * g for b in reversed(self.block))


class State:
    """The oracle's block-major State: fields with ghost widths."""

    def __init__(self, grid: Grid, ghosts):
        self.grid = grid
        self.ghosts = list(ghosts)
        self.h = lib.orc_state_create(grid.h, len(ghosts), (C.c_int * len(ghosts))(*ghosts))
        if not self.h:
            raise ValueError("invalid state (ghost wider than a block?)")

    def __del__(self):
        if getattr(self, "h", None):
            lib.orc_state_destroy(self.h)

    def get(self, f):
        g = self.ghosts[f]
        out = np.empty((self.grid.num_blocks(),) + self.grid.slab_shape(g), dtype=np.float64)
        lib.orc_state_get_field(self.h, f, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def set(self, f, data):
        arr = np.ascontiguousarray(data, dtype=np.float64)
        assert arr.size == self.grid.num_blocks() * self.grid.block_len(self.ghosts[f])
        lib.orc_state_set_field(self.h, f, arr.ctypes.data_as(C.POINTER(C.c_double)))

    def interior(self, f):
        g = self.ghosts[f]
        a = self.get(f)
        sl = (slice(None),) + tuple(slice(g, g + n) for n in reversed(self.grid.block))
        return np.ascontiguousarray(a[sl])

    def fill_ghosts(self, f):
        lib.orc_fill_ghosts_mirror(self.grid.h, self.h, f)

    def heat_run(self, f, kappa, t0, dt, steps, threads=1):
        return lib.orc_heat_run(self.grid.h, self.h, f, kappa, t0, dt, steps, threads)

    def modelc_run(self, params: Params, t0, dt, seed, steps, wiener, threads=1):
        return lib.orc_modelc_run(self.grid.h, self.h, C.byref(params), t0, dt, seed, steps, int(wiener), threads)

    def modelc_run_oriented(self, params: Params, theta_field, t0, dt, seed, steps, wiener, threads=1):
        return lib.orc_modelc_run_oriented(self.grid.h, self.h, C.byref(params), theta_field, t0, dt, seed, steps,
                                           int(wiener), threads)

    def heat_run_rk4(self, f, kappa, t0, dt, steps, threads=1):
        return lib.orc_heat_run_rk4(self.grid.h, self.h, f, kappa, t0, dt, steps, threads)

    def modelc_run_rk4(self, params: Params, t0, dt, steps, theta_field=-1, threads=1):
        return lib.orc_modelc_run_rk4(self.grid.h, self.h, C.byref(params), theta_field, t0, dt, steps, threads)

    def initialize_orientations(self, theta_field, grains):
        """grains: (x, y, radius, orientation) tuples."""
        arr = np.array([[g[0], g[1], g[2], g[3]] for g in grains], dtype=np.float64)
        lib.orc_modelc_initialize_orientations(self.grid.h, self.h, theta_field,
                                               arr.ctypes.data_as(C.POINTER(C.c_double)), len(grains))

    def modelc_drift(self, params: Params):
        n = self.grid.num_blocks() * self.grid.block_len(1)
        kp, ku = np.zeros(n), np.zeros(n)
        lib.orc_modelc_drift(self.grid.h, self.h, C.byref(params), kp.ctypes.data_as(C.POINTER(C.c_double)),
                             ku.ctypes.data_as(C.POINTER(C.c_double)))
        shape = (self.grid.num_blocks(),) + self.grid.slab_shape(1)
        return kp.reshape(shape), ku.reshape(shape)

    def initialize_grains(self, grains, u0):
        arr = np.array([[g[0], g[1], g[2], 0.0] for g in grains], dtype=np.float64)
        lib.orc_modelc_initialize_grains(self.grid.h, self.h, arr.ctypes.data_as(C.POINTER(C.c_double)), len(grains),
                                         u0)


def modelc_params(eps4=0.06, lam=3.19, d_thermal=None, noise=0.0, tol=1e-8, flux_tol=1e-8):
    """ModelC::new (phasefield.rs:100-116): d_thermal = A2 * lambda unless given."""
    return Params(eps4, lam, 0.6267 * lam if d_thermal is None else d_thermal, noise, tol, flux_tol)


# ----------------------------------------------------------------- AMR ---
def _amr_sigs():
    p, i64, u64, d = C.c_void_p, C.c_int64, C.c_uint64, C.c_double
    pd, pi64 = C.POINTER(C.c_double), C.POINTER(C.c_int64)
    sigs = {
        "orc_cluster": (i64, [C.c_int, pi64, i64, d, i64, pi64, i64]),
        "orc_amr_sim_create": (p, [pi64, pi64, pd, pd, C.POINTER(C.c_uint32), C.c_int, pi64, i64, C.c_int,
                                   C.POINTER(Params), d, C.c_int, u64, C.c_int, pd, C.POINTER(C.c_int)]),
        "orc_amr_sim_destroy": (None, [p]),
        "orc_amr_sim_set_threads": (None, [p, C.c_int]),
        "orc_amr_sim_num_blocks": (i64, [p]),
        "orc_amr_sim_num_levels": (C.c_int, [p]),
        "orc_amr_sim_epoch": (i64, [p]),
        "orc_amr_sim_patch": (None, [p, i64, pi64]),
        "orc_amr_sim_field_len": (i64, [p]),
        "orc_amr_sim_get_field": (None, [p, C.c_int, pd]),
        "orc_amr_sim_set_field": (None, [p, C.c_int, pd]),
        "orc_amr_sim_step": (d, [p, d, i64]),
        "orc_amr_sim_suggested_dt": (d, [p]),
        "orc_amr_sim_restrict": (None, [p, C.c_int]),
        "orc_amr_sim_fill_ghosts": (None, [p, C.c_int]),
        "orc_amr_sim_tag": (i64, [p, C.c_int, d, C.c_int, pi64, i64]),
        "orc_amr_sim_regrid_flags": (C.c_int, [p, pi64, i64, i64, d, i64]),
        "orc_amr_sim_cell_center": (None, [p, i64, pi64, pd]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


_amr_sigs()


def cluster(flags, efficiency, min_width):
    """Berger-Rigoutsos boxes [(lo, hi)] of flagged cells (list of tuples)."""
    D = len(flags[0]) if flags else 2
    arr = np.ascontiguousarray(np.array(flags, dtype=np.int64).reshape(-1, D) if flags else np.zeros((0, D), np.int64))
    cap = max(1, len(flags))
    out = np.zeros(cap * 2 * D, dtype=np.int64)
    n = lib.orc_cluster(D, arr.ctypes.data_as(C.POINTER(C.c_int64)), len(flags), efficiency, min_width,
                        out.ctypes.data_as(C.POINTER(C.c_int64)), cap)
    return [(tuple(out[i * 2 * D:i * 2 * D + D]), tuple(out[i * 2 * D + D:(i + 1) * 2 * D])) for i in range(n)]


class AmrSim:
    """The oracle's Simulation on an AmrGrid<2> (heat or Model C, subcycled
    or global dt, optional Berger-Oliger policy)."""

    def __init__(self, cells, block, h, ratios, patches=(), model="heat", params=None, kappa=0.7,
                 integrator="subcycling", seed=0, wiener=False, policy=None, origin=(0.0, 0.0)):
        pa = np.array([[lv, *lo, *hi] for lv, lo, hi in patches], dtype=np.int64).reshape(-1, 5)
        err = C.c_int(0)
        pol = None
        if policy is not None:
            pol = (C.c_double * 6)(policy["every"], policy["buffer"], policy["efficiency"], policy["min_width"],
                                   policy["threshold"], policy.get("field", 0))
        self.h = lib.orc_amr_sim_create(
            (C.c_int64 * 2)(*cells), (C.c_int64 * 2)(*block), (C.c_double * 2)(*origin), (C.c_double * 2)(h, h),
            (C.c_uint32 * len(ratios))(*ratios), len(ratios), pa.ctypes.data_as(C.POINTER(C.c_int64)), len(pa),
            0 if model == "heat" else 1, C.byref(params) if params is not None else None, kappa,
            0 if integrator == "subcycling" else 1, seed, int(wiener), pol, C.byref(err))
        self.err = err.value
        if not self.h:
            raise ValueError(f"AmrGrid::from_patches error {err.value}")
        self.nfields = 1 if model == "heat" else 2

    def __del__(self):
        if getattr(self, "h", None):
            lib.orc_amr_sim_destroy(self.h)

    def threads(self, n):
        lib.orc_amr_sim_set_threads(self.h, n)

    @property
    def num_blocks(self):
        return lib.orc_amr_sim_num_blocks(self.h)

    @property
    def num_levels(self):
        return lib.orc_amr_sim_num_levels(self.h)

    @property
    def epoch(self):
        return lib.orc_amr_sim_epoch(self.h)

    def patch(self, b):
        out = (C.c_int64 * 5)()
        lib.orc_amr_sim_patch(self.h, b, out)
        return int(out[0]), (int(out[1]), int(out[2])), (int(out[3]), int(out[4]))

    def patches(self):
        return [self.patch(b) for b in range(self.num_blocks)]

    def get(self, f):
        """List of per-block slabs, each (ny+2, nx+2)."""
        flat = np.empty(lib.orc_amr_sim_field_len(self.h))
        lib.orc_amr_sim_get_field(self.h, f, flat.ctypes.data_as(C.POINTER(C.c_double)))
        out, off = [], 0
        for lv, lo, hi in self.patches():
            nx, ny = hi[0] - lo[0], hi[1] - lo[1]
            n = (nx + 2) * (ny + 2)
            out.append(flat[off:off + n].reshape(ny + 2, nx + 2).copy())
            off += n
        return out

    def set(self, f, slabs):
        flat = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.float64).ravel() for s in slabs]))
        lib.orc_amr_sim_set_field(self.h, f, flat.ctypes.data_as(C.POINTER(C.c_double)))

    def step(self, dt, n=1):
        return lib.orc_amr_sim_step(self.h, dt, n)

    def suggested_dt(self):
        return lib.orc_amr_sim_suggested_dt(self.h)

    def restrict(self, f):
        lib.orc_amr_sim_restrict(self.h, f)

    def fill_ghosts(self, f):
        lib.orc_amr_sim_fill_ghosts(self.h, f)

    def tag(self, f, threshold, level):
        cap = 1 << 20
        out = np.zeros(2 * cap, dtype=np.int64)
        n = lib.orc_amr_sim_tag(self.h, f, threshold, level, out.ctypes.data_as(C.POINTER(C.c_int64)), cap)
        return [tuple(out[2 * i:2 * i + 2]) for i in range(n)]

    def regrid_flags(self, flags, buffer, efficiency, min_width):
        """Regrid now with these level-0 flags in place of the tagger; True
        when the hierarchy changed."""
        arr = np.ascontiguousarray(np.array(flags, dtype=np.int64).reshape(-1, 2))
        return bool(lib.orc_amr_sim_regrid_flags(self.h, arr.ctypes.data_as(C.POINTER(C.c_int64)), len(arr),
                                                 buffer, efficiency, min_width))

    def centers(self, b):
        """(xc, yc) arrays of the interior cell centres of block b, shape (ny, nx)."""
        lv, lo, hi = self.patch(b)
        nx, ny = hi[0] - lo[0], hi[1] - lo[1]
        xs = np.empty((ny, nx))
        ys = np.empty((ny, nx))
        out = (C.c_double * 2)()
        for j in range(ny):
            for i in range(nx):
                lib.orc_amr_sim_cell_center(self.h, b, (C.c_int64 * 2)(i, j), out)
                xs[j, i], ys[j, i] = out[0], out[1]
        return xs, ys
