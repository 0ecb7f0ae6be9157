"""Cell lists on the GPU against the oracle: bit-exact hashes, permutation, cell bounds and
gathered state (grid.cu:34-51, grid_gpu_green.cu:22-210, grid_gpu_rothlin.cu:28-250)."""
import numpy as np
import pytest

from conftest import bits_equal
from helpers import load_oracle, load_product, perturbed_scene

pytestmark = pytest.mark.gpu

GATHERED = ("pos", "vel", "fc", "h", "rho", "S", "eps_pl", "eps_pl_dot", "T", "fixed", "blanked", "tool_p",
            "pos_t", "vel_t", "rho_t", "S_t", "T_t")


def compare_cells(ctx, o, kind):
    assert np.array_equal(ctx.get("hash"), o.get("hash"))
    assert np.array_equal(ctx.get("idx"), o.get("idx"))
    ps, pe = ctx.cells()
    os_, oe = o.cells()
    if kind == 1:  # Rothlin: offsets everywhere
        assert np.array_equal(ps, os_) and np.array_equal(pe, oe)
    else:  # Green: start -1 on empty cells; end only meaningful where start != -1
        assert np.array_equal(ps, os_)
        occ = os_ != -1
        assert np.array_equal(pe[occ], oe[occ])
    for f in GATHERED + (("ft",) if kind == 0 else ()):
        assert bits_equal(ctx.get(f), o.get(f)), f


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("blank", [0.0, 0.05])
def test_cell_list_bitwise(mf, orc, kind, blank):
    st = perturbed_scene(mf, ny=12, seed=1, blank_frac=blank)
    ctx = load_product(mf, st, grid_kind=kind)
    o = load_oracle(orc, st, grid_kind=kind)
    rng = np.random.default_rng(3)
    dx = st["grid"][2]
    for rep in range(4):
        ctx.grid_build()
        assert o.L.orc_grid_update(o.s) == 0
        compare_cells(ctx, o, kind)
        # move particles up to 1.5 cells so that the next sort has movers in every direction
        pos = ctx.get("pos")
        pos += rng.uniform(-1.5, 1.5, pos.shape) * dx * (rng.random((pos.shape[0], 1)) < 0.2)
        ctx.set("pos", pos)
        o.set_field("pos", pos)
    st_ = ctx.status()
    assert st_["error_flags"] == 0 and st_["out_of_grid"] == 0


def test_crowded_cell_and_ragged_sizes(mf, orc):
    """Hundreds of particles in one cell (stable fix-up path) and N not a multiple of a block."""
    st = perturbed_scene(mf, ny=6, seed=2)
    N = st["N"]
    rng = np.random.default_rng(5)
    crowd = rng.choice(N, 301, replace=False)
    st["pos"][crowd] = st["pos"][crowd[0]] + rng.uniform(0, 1e-7, (301, 2))
    ctx = load_product(mf, st)
    o = load_oracle(orc, st)
    for _ in range(2):
        ctx.grid_build()
        o.L.orc_grid_update(o.s)
        compare_cells(ctx, o, 0)
    assert ctx.status()["max_cell_occupancy"] >= 301


def test_out_of_grid_is_clamped_and_counted(mf, orc):
    st = perturbed_scene(mf, ny=6, seed=3)
    bbmin, bbmax, h = st["grid"]
    st["pos"][0] = (bbmin[0] - 10 * h, bbmin[1] - 10 * h)
    st["pos"][1] = (bbmax[0] + 10 * h, bbmax[1] + 10 * h)
    ctx = load_product(mf, st)
    o = load_oracle(orc, st)
    ctx.grid_build()
    o.L.orc_grid_update(o.s)
    compare_cells(ctx, o, 0)
    assert ctx.status()["out_of_grid"] == o.L.orc_out_of_grid(o.s) == 2


@pytest.mark.parametrize("kind", [0, 1])
def test_adaptive_grid(mf, orc, kind):
    """update_geometry (grid.cu:97-136): box and cell size from the particles every sort."""
    st = perturbed_scene(mf, ny=8, seed=4)
    ctx = load_product(mf, st, grid_kind=kind)
    o = load_oracle(orc, st, grid_kind=kind)
    max_cell = 4 * st["N"]
    ctx.grid_adaptive(kind, max_cell)
    o.L.orc_set_grid_adaptive(o.s, kind, max_cell)
    for _ in range(2):
        ctx.grid_build()
        assert o.L.orc_grid_update(o.s) == 0
        g1, g2 = ctx.geometry(), o.geometry()
        for k in ("nx", "ny", "num_cell"):
            assert g1[k] == g2[k], k
        for k in ("bbmin_x", "bbmin_y", "bbmax_x", "bbmax_y", "dx"):
            assert bits_equal(g1[k], g2[k]), k
        compare_cells(ctx, o, kind)


def test_single_particle(mf, orc):
    st = perturbed_scene(mf, ny=6, seed=5)
    keep = np.array([int(np.argmax(st["tool_p"] == 0))])
    small = {k: (v[keep] if isinstance(v, np.ndarray) and v.shape[:1] == (st["N"],) else v) for k, v in st.items()}
    small["N"] = 1
    ctx = load_product(mf, small)
    o = load_oracle(orc, small)
    ctx.grid_build()
    o.L.orc_grid_update(o.s)
    compare_cells(ctx, o, 0)
