"""mf_cells_build_noalloc: the cell list for callers that cannot allocate device memory.

Such a caller (a host that reserves all device memory up front and allows no driver
allocation during a run, or a binding that only passes device pointers) gets the same
hash, stable permutation and cell bounds as mf_grid_build, computed in a fixed scratch
array inside the library. These tests allocate the input/output buffers themselves (the
caller's side) and check the integer outputs for equality: two calls in a row against
mf_grid_build, and against the oracle's cell lists at the ~150k-particle benchmark geometry,
at the entry point's particle and cell limits and on one crowded cell. The file is named so
that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import load_product, perturbed_scene

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 1 << 19
MAX_CELLS = 1 << 21


class NoallocStatus(C.Structure):
    _fields_ = [("out_of_grid", C.c_ulonglong), ("error_flags", C.c_ulonglong),
                ("max_cell_occupancy", C.c_ulonglong)]


def _fn(mf):
    f = mf.lib().mf_cells_build_noalloc
    f.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int] + [C.c_void_p] * 6
    f.restype = C.c_int
    return f


def _noalloc_cells(mf, torch, pos, geo):
    """Run the allocation-free entry point on positions (N x 2) with caller-owned buffers;
    returns (hash, idx, cell_start, cell_end, status)."""
    N = pos.shape[0]
    nc = geo["num_cell"]
    d_pos = torch.from_numpy(np.ascontiguousarray(pos, dtype=np.float64)).cuda()
    d_hash = torch.full((N,), -7, dtype=torch.int32, device="cuda")
    d_idx = torch.full((N,), -7, dtype=torch.int32, device="cuda")
    d_start = torch.full((nc,), -7, dtype=torch.int32, device="cuda")
    d_end = torch.full((nc,), -7, dtype=torch.int32, device="cuda")
    d_status = torch.full((3,), -1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = _fn(mf)(d_pos.data_ptr(), N, geo["bbmin_x"], geo["bbmin_y"], geo["dx"], geo["nx"], geo["ny"],
                 d_hash.data_ptr(), d_idx.data_ptr(), d_start.data_ptr(), d_end.data_ptr(), d_status.data_ptr(),
                 stream.cuda_stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    s = d_status.cpu().numpy()
    status = {"out_of_grid": int(s[0]), "error_flags": int(s[1]), "max_cell_occupancy": int(s[2])}
    return d_hash.cpu().numpy(), d_idx.cpu().numpy(), d_start.cpu().numpy(), d_end.cpu().numpy(), status


def _grid_build_cells(mf, st, pos):
    """The existing entry point: mf_grid_build on a context holding the same positions."""
    ctx = load_product(mf, dict(st, pos=pos))
    geo = ctx.geometry()
    ctx.grid_build()
    start, end = ctx.cells()
    out = ctx.get("hash"), ctx.get("idx"), start, end
    ctx.close()
    return geo, out


def _oracle_cells(orc, pos, bbmin, bbmax, h):
    """The oracle's cell list (assign_hashes + stable sort_by_key + cell start/end of
    grid_gpu_green) for positions on a locked grid; returns geometry and outputs."""
    N = pos.shape[0]
    o = orc.Oracle(N)
    o.set_field("pos", pos)
    o.set_field("h", np.full(N, h))
    o.set_field("rho", np.ones(N))
    o.L.orc_set_grid_locked(o.s, 0, bbmin[0], bbmin[1], bbmax[0], bbmax[1], h)
    assert o.L.orc_grid_update(o.s) == 0
    start, end = o.cells()
    return o.geometry(), (o.get("hash"), o.get("idx"), start, end), int(o.L.orc_out_of_grid(o.s))


def _assert_same_cells(got, expected):
    hash_, idx, start, end = got[:4]
    e_hash, e_idx, e_start, e_end = expected
    assert np.array_equal(hash_, e_hash), "hash"
    assert np.array_equal(idx, e_idx), "idx"
    assert np.array_equal(start, e_start), "cell_start"
    occupied = e_start != -1  # grid_gpu_green leaves cell_end stale on empty cells
    assert np.array_equal(end[occupied], e_end[occupied]), "cell_end"
    assert np.all(end[~occupied] == -1)


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
        assert got[4]["out_of_grid"] == 0 and got[4]["error_flags"] == 0
    # the second call reused the scratch of the first: still no leftovers
    assert np.array_equal(np.sort(got[1]), np.arange(pos2.shape[0]))


def test_noalloc_matches_oracle_at_benchmark_geometry(mf, orc):
    """The ~150k-particle cut (714 x 214 lattice + tool particles, ~350k cells, ~170 scan
    tiles): equal to the oracle's cell lists, before and after a random displacement."""
    import torch
    import bench

    p, _, _ = bench.config_params(mf, "c2")
    sc = mf.Scene.from_params(p)
    s = sc.s
    bbmin, bbmax, h = tuple(s.grid_bbmin), tuple(s.grid_bbmax), s.grid_h
    rng = np.random.default_rng(5)
    pos0 = sc.array("pos").copy()
    for pos in (pos0, pos0 + rng.uniform(-0.6, 0.6, pos0.shape) * h):
        geo, expected, oog = _oracle_cells(orc, pos, bbmin, bbmax, h)
        assert oog == 0
        assert geo["num_cell"] > 300_000
        got = _noalloc_cells(mf, torch, pos, geo)
        _assert_same_cells(got, expected)
        assert got[4]["out_of_grid"] == 0 and got[4]["error_flags"] == 0
        assert got[4]["max_cell_occupancy"] == int(np.bincount(expected[0]).max())


def test_noalloc_at_its_limits_matches_oracle(mf, orc):
    """MF_NOALLOC_MAX_PARTICLES particles on a grid of MF_NOALLOC_MAX_CELLS cells."""
    import torch

    h = 1.0 / 1024.0
    bbmin, bbmax = (0.0, 0.0), (2.0 - 4e-6, 1.0 - 4e-6)  # nx = 2048, ny = 1024 after the margins
    rng = np.random.default_rng(11)
    pos = np.stack([rng.uniform(0.0, bbmax[0], MAX_PARTICLES), rng.uniform(0.0, bbmax[1], MAX_PARTICLES)], axis=1)
    geo, expected, oog = _oracle_cells(orc, pos, bbmin, bbmax, h)
    assert (geo["nx"], geo["ny"], geo["num_cell"]) == (2048, 1024, MAX_CELLS)
    assert oog == 0
    got = _noalloc_cells(mf, torch, pos, geo)
    _assert_same_cells(got, expected)
    assert got[4]["error_flags"] == 0


def test_noalloc_crowded_cell_and_clamped_particle(mf, orc):
    """400 of 700 particles in one cell (the stable in-cell order over a long cell), and one
    particle left of the grid: clamped into cell 0 and counted, as the oracle does."""
    import torch

    h = 0.1
    bbmin, bbmax = (0.0, 0.0), (0.8, 0.8)
    rng = np.random.default_rng(3)
    pos = rng.uniform(0.0, 0.8, (700, 2))
    crowd = rng.permutation(700)[:400]
    pos[crowd] = 0.33 + rng.uniform(0.0, 0.05, (400, 2))
    pos[17] = (-0.5, 0.2)
    geo, expected, oog = _oracle_cells(orc, pos, bbmin, bbmax, h)
    assert oog == 1
    got = _noalloc_cells(mf, torch, pos, geo)
    _assert_same_cells(got, expected)
    assert got[4]["out_of_grid"] == 1
    assert got[4]["max_cell_occupancy"] >= 400


def test_noalloc_rejects_bad_sizes_and_misaligned_pointers(mf):
    import torch

    f = _fn(mf)
    too_many = MAX_PARTICLES + 1
    assert f(None, too_many, 0.0, 0.0, 1.0, 4, 4, None, None, None, None, None, None) == -4
    assert f(None, 16, 0.0, 0.0, 1.0, 1 << 11, (1 << 10) + 1, None, None, None, None, None, None) == -4
    assert f(None, 0, 0.0, 0.0, 1.0, 4, 4, None, None, None, None, None, None) == -1
    # positions 8 bytes off a 16-byte boundary: refused before any launch
    buf = torch.zeros(2 * 16 + 2, dtype=torch.float64, device="cuda")
    ints = torch.zeros(64, dtype=torch.int32, device="cuda")
    p = ints.data_ptr()
    assert f(buf.data_ptr() + 8, 16, 0.0, 0.0, 1.0, 4, 4, p, p + 64, p + 128, p + 192, None, None) == -1
    assert f(buf.data_ptr(), 16, 0.0, 0.0, 1.0, 4, 4, p + 2, p + 64, p + 128, p + 192, None, None) == -1
    torch.cuda.synchronize()
