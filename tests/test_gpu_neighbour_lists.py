"""Neighbour lists of the mixed form (opt-in, MF_OPT_NEIGHBOUR_LISTS) against the mixed form
that sorts every step (the default).

With neighbour lists the cell list is sorted only on the steps where some particle would
otherwise be more than 0.45 skin from where its list was built; in between, each particle
visits the candidates it listed at the last sort, in that sort's order. A sorting step's
list holds the 5x5 window's in-support candidates in the window's order, and while no
particle changes cell a later step sees the order, the cells and the neighbour set of the
step that sorts every step: both give the same bits. Once particles cross cells only the
FP32 summation order (and the cell each FP32 coordinate is taken relative to) differs.
"""
import numpy as np
import pytest

from conftest import rel_err
from helpers import load_product, perturbed_scene

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "rho", "S", "T", "eps_pl", "eps_pl_dot", "fc", "ft", "pos_t", "vel_t", "S_t", "rho_t", "T_t")


def by_id(ctx, f):
    return ctx.get(f)[np.argsort(ctx.get("id"))]


def pair(mf, st, **kw):
    a = load_product(mf, st, precision=mf.PRECISION_MIXED, flags=mf.OPT_NEIGHBOUR_LISTS, **kw)
    b = load_product(mf, st, precision=mf.PRECISION_MIXED, flags=mf.OPT_SORT_EVERY_STEP, **kw)
    return a, b


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("blank_frac", [0.0, 0.05])
def test_lists_equal_sorting_every_step(mf, blank_frac, fused):
    """A step on lists in which no particle changed cell: the same bits as sorting every step."""
    # the tool at rest and not in contact: slow particles, no sort after the first
    st = perturbed_scene(mf, ny=12, seed=61, blank_frac=blank_frac, tool_push_dx=0.0)
    st["tool"].vel[0] = st["tool"].vel[1] = 0.0
    a, b = pair(mf, st)
    if fused:
        a.set_flags(mf.OPT_NEIGHBOUR_LISTS | mf.OPT_FUSED_PREDICTOR)
    a.step(1)
    b.step(1)
    cells0 = by_id(b, "hash")
    a.step(1)
    b.step(1)
    sa, sb = a.status(), b.status()
    assert sb["sorts"] == 2 and sa["sorts"] == 1, (sa["sorts"], sb["sorts"])
    assert sa["error_flags"] == 0 and sb["error_flags"] == 0
    # no particle changed cell in the form that sorts every step, so its order and
    # neighbour sets are those of the lists
    assert np.array_equal(cells0, by_id(b, "hash"))
    assert np.array_equal(by_id(a, "hash"), cells0)
    assert np.array_equal(by_id(a, "blanked"), by_id(b, "blanked"))
    for f in FIELDS:
        x, y = by_id(a, f), by_id(b, f)
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), f
    assert np.array_equal(a.force_log(), b.force_log())


def test_thin_skin_sorts_every_step(mf):
    """A skin below one step's motion: every step sorts and rebuilds the lists, so the run is
    the one of the form that sorts every step, bit for bit, with the tool cutting into the
    workpiece and some particles blanked."""
    st = perturbed_scene(mf, ny=12, seed=63, blank_frac=0.02)
    a, b = pair(mf, st)
    a.set_neighbour_skin(1e-18)
    a.step(8)
    b.step(8)
    sa = a.status()
    assert sa["sorts"] == 8 and sa["error_flags"] == 0, (sa["sorts"], sa["error_flags"])
    assert np.array_equal(a.get("id"), b.get("id"))
    for f in FIELDS + ("blanked",):
        x, y = a.get(f), b.get(f)
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), f
    assert np.array_equal(a.force_log(), b.force_log())


@pytest.mark.parametrize("fused", [False, True])
def test_lists_close_to_sorting_every_step(mf, fused):
    """The tool pushed into the workpiece: fast particles that cross cells and force sorts;
    only the FP32 summation order differs."""
    st = perturbed_scene(mf, ny=12, seed=65, blank_frac=0.02)
    a, b = pair(mf, st)
    if fused:
        a.set_flags(mf.OPT_NEIGHBOUR_LISTS | mf.OPT_FUSED_PREDICTOR)
    a.step(40)
    b.step(40)
    sa = a.status()
    assert sa["error_flags"] == 0
    assert np.array_equal(by_id(a, "blanked"), by_id(b, "blanked"))
    for f in FIELDS:
        x, y = by_id(a, f), by_id(b, f)
        assert rel_err(x, y) < 1e-4, (f, rel_err(x, y), sa["sorts"])


def test_lists_track_sorting_every_step_long(mf):
    """Many steps with the tool cutting: particles cross cells and the lists are rebuilt."""
    st = perturbed_scene(mf, ny=12, seed=62, tool_push_dx=1.0)
    a, b = pair(mf, st)
    a.set_neighbour_skin(0.02 * st["grid"][2])  # a thin skin: several sorts in the run
    a.step(400)
    b.step(400)
    sa = a.status()
    assert sa["error_flags"] == 0
    assert 2 <= sa["sorts"] < 400, sa["sorts"]
    assert np.array_equal(by_id(a, "blanked"), by_id(b, "blanked"))
    pa, pb = by_id(a, "pos"), by_id(b, "pos")
    assert np.abs(pa - pb).max() / st["grid"][2] < 1e-5, np.abs(pa - pb).max() / st["grid"][2]
    for f in ("vel", "rho", "S", "T", "eps_pl"):
        assert rel_err(by_id(a, f), by_id(b, f)) < 1e-3, (f, rel_err(by_id(a, f), by_id(b, f)), sa["sorts"])
    fa, fb = a.force_log(), b.force_log()
    assert rel_err(fa.mean(axis=0), fb.mean(axis=0)) < 1e-4
    # the fields a list step without a sort does not rewrite (order, numbers, smoothing lengths)
    # after sorts and runs of steps without one: every particle still carries its own
    assert np.array_equal(np.sort(a.get("id")), np.arange(st["N"]))
    assert np.array_equal(by_id(a, "h"), by_id(b, "h"))
    assert np.array_equal(by_id(a, "tool_p"), by_id(b, "tool_p"))


def test_sorts_every_step_outside_list_mode(mf):
    st = perturbed_scene(mf, ny=10, seed=64)
    for kw in ({"precision": mf.PRECISION_FP64}, {"precision": mf.PRECISION_MIXED},
               {"precision": mf.PRECISION_MIXED, "thermal_solver": 1, "flags": mf.OPT_NEIGHBOUR_LISTS}):
        c = load_product(mf, st, **kw)
        c.step(5)
        assert c.status()["sorts"] == 5, kw


def test_large_skin_is_limited(mf):
    """A skin of ten cells is limited to half a cell: the lists stay complete and below their
    64 entries (no error flag), and the run follows the form that sorts every step."""
    st = perturbed_scene(mf, ny=12, seed=66, blank_frac=0.02)
    a, b = pair(mf, st)
    a.set_neighbour_skin(10.0 * st["grid"][2])
    a.step(30)
    b.step(30)
    sa = a.status()
    assert sa["error_flags"] == 0, sa["error_flags"]
    assert sa["sorts"] < 30
    assert np.array_equal(by_id(a, "blanked"), by_id(b, "blanked"))
    for f in FIELDS:
        x, y = by_id(a, f), by_id(b, f)
        assert rel_err(x, y) < 1e-4, (f, rel_err(x, y), sa["sorts"])


@pytest.mark.parametrize("fused", [False, True])
def test_lists_hold_every_in_support_pair(mf, fused):
    """The list invariant checked by brute force after every step (mf_list_check): with the
    scene's random velocities 30 times faster (the fastest particles reach 0.45 skin in a few
    steps) and the tool cutting, the lists are reused up to their limit and rebuilt many times;
    every unblanked pair closer than 2 h_i in the pair records must be in the lists."""
    # (the tool one cell into the workpiece: where tool and workpiece particles overlap the
    # candidates within 2h + skin double, and three cells of overlap would bring them near the
    # 64 entries of a row)
    st = perturbed_scene(mf, ny=12, seed=68, blank_frac=0.02, tool_push_dx=1.0)
    st["vel"] = st["vel"] * 30.0
    flags = mf.OPT_NEIGHBOUR_LISTS | (mf.OPT_FUSED_PREDICTOR if fused else 0)
    ctx = load_product(mf, st, precision=mf.PRECISION_MIXED, flags=flags)
    checked = 0
    for k in range(80):
        ctx.step(1)
        r = ctx.list_check()
        live = int((ctx.get("blanked") == 0.0).sum())
        assert r["pairs"] > 10 * live, (k, r, live)  # ~24 in-support neighbours per particle
        if not r["stale"]:
            assert r["missing"] == 0, (k, r)
            checked += 1
    s = ctx.status()
    assert s["error_flags"] == 0
    assert 2 <= s["sorts"] < 80, s["sorts"]
    assert checked >= (80 if not fused else 40), checked


def test_list_check_needs_a_list_step(mf):
    st = perturbed_scene(mf, ny=8, seed=69)
    ctx = load_product(mf, st, precision=mf.PRECISION_MIXED)  # sorts every step: no lists
    ctx.step(2)
    with pytest.raises(mf.MfError):
        ctx.list_check()
