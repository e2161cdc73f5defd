"""The C-ABI library loads and exports every entry point include/*.h declares (CPU)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(lg_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import legendre_b200._native as N
    lib = ctypes.CDLL(str(N._LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert len(declared_symbols()) >= 20


def test_binding_covers_every_declared_symbol():
    import legendre_b200._native as N
    assert set(declared_symbols()) <= set(N.exported_symbols())


def test_abi_version():
    import legendre_b200._native as N
    assert N.lib.lg_abi_version() == 1


def test_null_arguments_are_rejected_without_a_device():
    import legendre_b200._native as N
    assert N.lib.lg_ctx_create(0, None, None) == N.LG_ERR_INVALID
    assert N.lib.lg_sync(None, 0) == N.LG_ERR_INVALID
    assert N.lib.lg_state_destroy(None) == N.LG_ERR_INVALID
    assert N.lib.lg_last_error(None) == b"null context"


def test_grid_validation_mirrors_the_reference():
    # CartesianGrid::new errors (cartesian.rs:48-82; tests/framework.rs:30-46)
    # on the host mirror
    import pytest
    from legendre_b200 import CartesianGrid, GridError
    with pytest.raises(GridError):
        CartesianGrid([10], [3], [0.0], [1.0])
    with pytest.raises(GridError):
        CartesianGrid([0], [1], [0.0], [1.0])
    with pytest.raises(GridError):
        CartesianGrid([4], [2], [0.0], [0.0])
    g = CartesianGrid([4, 4], [2, 2], [0.0, 0.0], [1.0, 1.0]).with_periodic([True, False])
    assert g.face_neighbor(0, 0, -1) == 1 and g.face_neighbor(0, 1, -1) is None


def test_host_grid_matches_oracle(orc):
    from legendre_b200 import CartesianGrid
    for cells, block, per in [([12, 8], [4, 4], [True, False]), ([6, 6, 6], [2, 3, 6], [True, True, False]),
                              ([8], [8], [True])]:
        D = len(cells)
        a = CartesianGrid(cells, block, [0.0] * D, [0.5] * D).with_periodic(per)
        b = orc.Grid(cells, block, [0.0] * D, [0.5] * D, per)
        for blk in range(a.num_blocks()):
            for d in range(D):
                for s in (-1, 1):
                    assert a.face_neighbor(blk, d, s) == b.face_neighbor(blk, d, s)
            assert a.cell_center(blk, [1] * D) == b.cell_center(blk, [1] * D)


def test_seed_positions_follow_the_example():
    # examples/model_c.rs:175-206
    from legendre_b200 import seed_positions
    from legendre_b200.rng import mix_key, unit_open
    g = seed_positions(4096, 0.4, 16, 42, radius=8.0)
    margin = 16.0
    span = 4096 * 0.4 - 2.0 * margin
    assert len(g) == 16
    assert g[3].center[0] == margin + unit_open(mix_key(42, [3, 0])) * span
    one = seed_positions(630, 0.4, 1, 42)
    assert one[0].center == (0.4, 0.4) and one[0].radius == 4.0


def test_every_entry_point_rejects_null_handles_without_a_device():
    # each entry point checks its handle and output pointers before any CUDA
    # call: with null pointers and zero counts it returns LG_ERR_INVALID (the
    # two counters -1, lg_last_error its fixed text)
    import ctypes as C
    import legendre_b200._native as N
    special = {"lg_abi_version": 1, "lg_ctx_kernel_launches": -1, "lg_grid_num_blocks": -1,
               "lg_last_error": b"null context"}
    for name, (_res, args) in N._SIGS.items():
        vals = []
        for a in args:
            if a in (C.c_int, C.c_int64, C.c_uint64, C.c_uint32):
                vals.append(0)
            elif a is C.c_double:
                vals.append(0.0)
            else:  # a pointer or handle
                vals.append(None)
        got = getattr(N.lib, name)(*vals)
        assert got == special.get(name, N.LG_ERR_INVALID), name
