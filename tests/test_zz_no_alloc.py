"""mf_cells_build_noalloc: the cell list for callers that cannot allocate device memory.

Such a caller (a host that reserves all device memory up front and allows no driver
allocation during a run, or a binding that only passes device pointers) gets the same
hash, stable permutation and cell bounds as mf_grid_build, computed in a fixed scratch
array inside the library. This test allocates its own input/output buffers (the caller's
side) and checks two calls in a row against mf_grid_build; integer outputs must be equal.
The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import load_product, perturbed_scene

pytestmark = pytest.mark.gpu


def _fn(mf):
    f = mf.lib().mf_cells_build_noalloc
    f.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int] + [C.c_void_p] * 5
    f.restype = C.c_int
    return f


def _noalloc_cells(mf, torch, pos, geo):
    """Run the allocation-free entry point on positions (N x 2) with caller-owned buffers."""
    N = pos.shape[0]
    nc = geo["num_cell"]
    d_pos = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
    d_hash = torch.full((N,), -7, dtype=torch.int32, device="cuda")
    d_idx = torch.full((N,), -7, dtype=torch.int32, device="cuda")
    d_start = torch.full((nc,), -7, dtype=torch.int32, device="cuda")
    d_end = torch.full((nc,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = _fn(mf)(d_pos.data_ptr(), N, geo["bbmin_x"], geo["bbmin_y"], geo["dx"], geo["nx"], geo["ny"],
                 d_hash.data_ptr(), d_idx.data_ptr(), d_start.data_ptr(), d_end.data_ptr(), stream.cuda_stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return d_hash.cpu().numpy(), d_idx.cpu().numpy(), d_start.cpu().numpy(), d_end.cpu().numpy()


def _grid_build_cells(mf, st, pos):
    """The existing entry point: mf_grid_build on a context holding the same positions."""
    ctx = load_product(mf, dict(st, pos=pos))
    geo = ctx.geometry()
    ctx.grid_build()
    start, end = ctx.cells()
    out = ctx.get("hash"), ctx.get("idx"), start, end
    ctx.close()
    return geo, out


def test_noalloc_matches_grid_build_on_two_calls(mf):
    import torch

    st = perturbed_scene(mf, ny=14, seed=21)
    rng = np.random.default_rng(22)
    pos1 = st["pos"].copy()
    # second input: particles moved up to a cell in every direction
    pos2 = pos1 + rng.uniform(-1.0, 1.0, pos1.shape) * st["grid"][2] * (rng.random((pos1.shape[0], 1)) < 0.3)
    for pos in (pos1, pos2):
        geo, expected = _grid_build_cells(mf, st, pos)
        got = _noalloc_cells(mf, torch, pos, geo)
        for name, a, b in zip(("hash", "idx", "cell_start", "cell_end"), got, expected):
            assert np.array_equal(a, b), name
    # the second call reused the scratch of the first: still no leftovers
    assert np.array_equal(np.sort(got[1]), np.arange(pos2.shape[0]))


def test_noalloc_rejects_sizes_beyond_its_maximum(mf):
    f = _fn(mf)
    too_many = (1 << 19) + 1
    assert f(None, too_many, 0.0, 0.0, 1.0, 4, 4, None, None, None, None, None) == -4
    assert f(None, 16, 0.0, 0.0, 1.0, 1 << 11, (1 << 10) + 1, None, None, None, None, None) == -4
    assert f(None, 0, 0.0, 0.0, 1.0, 4, 4, None, None, None, None, None) == -1
