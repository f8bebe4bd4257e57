"""The allocation-free marching-cubes entry point, for callers that cannot let a library allocate
device memory (a solver budgeting its own pool, a time-stepping loop that cannot afford a
cudaMalloc mid-step). It must produce exactly what the handle-based entry point produces from the
same nodal field, call after call, although both share one static scratch array.

Collected last (file name), so a failure here comes after every other test has run."""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import cc, assert_cells_bitwise

pytestmark = pytest.mark.gpu
_lib = __import__("cutcell_b200._lib", fromlist=["_lib"])
_cache = __import__("cutcell_b200.cache", fromlist=["cache"])


def _noalloc(grid, phi, table, dtype):
    """One call of cc_mc_cells_from_phi_noalloc through the C ABI; returns host columns."""
    L = _lib.load()
    dev = torch.cuda.current_device()
    cols = _cache.CellColumns(grid.ncell, 3, dtype, torch.device("cuda", dev))
    gs = _cache.grid_struct(grid)
    cs = cols.struct()
    blob = C.create_string_buffer(table, len(table))
    prec = 1 if dtype == torch.float64 else 0
    stream = torch.cuda.current_stream().cuda_stream
    st = L.cc_mc_cells_from_phi_noalloc(dev, prec, C.byref(gs), blob, len(table), C.c_void_p(phi.data_ptr()),
                                        C.byref(cs), C.c_void_p(stream))
    assert st == _lib.CC_OK, _lib.last_error()
    torch.cuda.synchronize()
    return cols.to_host()


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_noalloc_matches_handle_entry_point_twice(dtype):
    table = cc.mc_tables.project_table()
    cases = [
        # a TMA-addressable grid (x extent a multiple of 16) and one that is not
        (cc.workloads.csg_grid(64), cc.workloads.csg_body(5)),
        (cc.CartesianGrid((-1.2, -0.9, -1.1), (35, 33, 31), (0.07, 0.06, 0.075)),
         cc.Union(cc.Sphere((0.1, 0.0, -0.1), 0.7), cc.Box((-0.2, 0.1, 0.3), (0.4, 0.3, 0.2)))),
    ]
    for grid, body in cases:
        ref = cc.update_cache(cc.allocate_cache(grid, cc.MarchingCubesCutCell(), dtype=dtype), body, grid)
        # two calls in a row: the first may copy the table into the shared array, the second finds
        # it there; both must give what the handle-based entry point gives
        for call in range(2):
            got = _noalloc(grid, ref.phi, table, dtype)
            assert_cells_bitwise(got, ref.to_host(), label=f"noalloc {grid.n} call {call + 1}")
        assert (got["kind"] == 2).sum() > 100


def test_noalloc_rejects_oversized_grid():
    L = _lib.load()
    g = cc.CartesianGrid((0.0, 0.0, 0.0), (256, 256, 256), (1.0, 1.0, 1.0))  # 2^24 cells > 2^23
    gs = _cache.grid_struct(g)
    cols = _cache.CellColumns(1, 3, torch.float32, torch.device("cuda"))
    cs = cols.struct()
    table = cc.mc_tables.project_table()
    blob = C.create_string_buffer(table, len(table))
    phi = torch.zeros(1, device="cuda")
    st = L.cc_mc_cells_from_phi_noalloc(torch.cuda.current_device(), 0, C.byref(gs), blob, len(table),
                                        C.c_void_p(phi.data_ptr()), C.byref(cs), None)
    assert st == _lib.CC_TOO_LARGE
    assert "at most 8388608 cells" in _lib.last_error()
