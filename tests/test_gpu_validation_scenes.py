"""The reference's validation scenes stepped on the GPU against the oracle.

  * rings (setup_rings, benchmarks.cpp:161-253): two rubber-like rings, 0.002 apart, moving at
    +-200 toward each other; locked Green grid; no plasticity, no heat, no tool;
  * impact (setup_impact, benchmarks.cpp:23-159): a steel disc at 1000 against a wall fixed at
    top and bottom; adaptive grid (Green, as the scene builds it, and Rothlin); Johnson-Cook
    plasticity; no heat, no tool.

Chained single-step parity: before every step the product's whole state (in its current array
order) is loaded into a fresh oracle, both take one step stage by stage, and the results are
compared, so that the comparison follows the scene's evolving state (the collision, the impact
and its plastic zone) without the chaotic growth of differences over many steps. The artificial
stress R comes from the reference's atan2f/cosf/sinf in float, whose CUDA and glibc results
differ by a few float ulps: it is compared at 1e-5 and the oracle continues from the product's,
as in the plain step's stage tests. Then (norm-wise) rates 1e-12 and state 1e-11, eps_pl_dot
1e-7 (the reference rounds the plastic multiplier to float). Cell order, blanking and the grid's
geometry are compared exactly.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import bits_equal, rel_err

pytestmark = pytest.mark.gpu

# (idx too: the Rothlin grid carries it through every sort as the particle's number)
LOADED = ("pos", "vel", "rho", "T", "h", "fixed", "tool_p", "S", "eps_pl", "eps_pl_dot", "fc", "ft", "n",
          "pos_t", "vel_t", "rho_t", "S_t", "T_t", "blanked", "idx")
STATE = ("pos", "vel", "S", "rho", "T", "eps_pl", "eps_pl_dot")
RATES = ("pos_t", "vel_t", "S_t", "rho_t")
FLOAT_ROUNDED = {"eps_pl_dot": 1e-7}


def oracle_from(orc, ctx, sc, grid_kind):
    """A fresh oracle holding the product's current state and the scene's constants and grid."""
    s = sc.s
    o = orc.Oracle(sc.N)
    for k in LOADED:
        o.set_field(k, ctx.get(k))
    if s.grid_max_cell > 0:
        o.L.orc_set_grid_adaptive(o.s, grid_kind, s.grid_max_cell)
    else:
        o.L.orc_set_grid_locked(o.s, grid_kind, s.grid_bbmin[0], s.grid_bbmin[1], s.grid_bbmax[0], s.grid_bbmax[1],
                                s.grid_h)
    phys = orc.OrcPhys(*[getattr(s.phys, f) for f, _ in orc.OrcPhys._fields_])
    corr = orc.OrcCorr(*[getattr(s.corr, f) for f, _ in orc.OrcCorr._fields_])
    joco = orc.OrcJoco(*[getattr(s.joco, f) for f, _ in orc.OrcJoco._fields_])
    tw = orc.OrcTrml(*[getattr(s.trml_wp, f) for f, _ in orc.OrcTrml._fields_])
    tt = orc.OrcTrml(*[getattr(s.trml_tool, f) for f, _ in orc.OrcTrml._fields_])
    o.L.orc_set_constants(o.s, C.byref(phys), C.byref(corr), C.byref(joco) if s.has_joco else None, C.byref(tw),
                          C.byref(tt))
    o.L.orc_set_options(o.s, 0, 0)
    o.L.orc_set_dt(o.s, s.dt)
    o.L.orc_set_tool(o.s, None)
    o._keep = (phys, corr, joco, tw, tt)
    return o


def compare(ctx, o, fields, tol, mask):
    for f in fields:
        a, b = ctx.get(f)[mask], o.get(f)[mask]
        assert np.isfinite(a).all() == np.isfinite(b).all(), f
        e = rel_err(a, b)
        assert e <= max(tol, FLOAT_ROUNDED.get(f, 0.0)), (f, e)


@pytest.mark.parametrize("kind,nbox,grid_kind,steps", [("rings", 21, 0, 20), ("impact", 17, 0, 20),
                                                        ("impact", 17, 1, 12)])
def test_validation_scene_steps_against_oracle(mf, orc, kind, nbox, grid_kind, steps):
    sc = getattr(mf.Scene, kind)(nbox)
    ctx = mf.Context(0)
    ctx.upload_scene(sc, grid_kind)
    r_steps = 0
    for k in range(steps):
        o = oracle_from(orc, ctx, sc, grid_kind)
        ctx.stage(0)  # cell list
        ctx.stage(1)  # predictor, EOS, artificial stress
        assert o.L.orc_grid_update(o.s) == 0, k
        o.L.orc_stage_predict(o.s)
        R = ctx.get("R")
        assert rel_err(R, o.get("R")) <= 1e-5, k
        r_steps += int(np.any(R != 0.0))
        o.set_field("R", R)
        ctx.stage(2)  # pair sums and rates
        o.L.orc_stage_interact(o.s)
        o.L.orc_stage_rates(o.s)
        ctx.stage(3)  # corrector .. boundary conditions, return map
        o.L.orc_stage_finish(o.s)
        assert np.array_equal(ctx.get("idx"), o.get("idx")), k
        blanked = ctx.get("blanked")
        assert np.array_equal(blanked, o.get("blanked")), k
        if sc.s.grid_max_cell > 0:  # the box and cell size update_geometry found (grid.cu:97-136)
            g1, g2 = ctx.geometry(), o.geometry()
            assert (g1["nx"], g1["ny"], g1["num_cell"]) == (g2["nx"], g2["ny"], g2["num_cell"]), k
            assert bits_equal([g1[f] for f in ("bbmin_x", "bbmin_y", "dx")],
                              [g2[f] for f in ("bbmin_x", "bbmin_y", "dx")]), k
        compare(ctx, o, RATES, 1e-12, blanked == 0.0)
        compare(ctx, o, STATE, 1e-11, blanked == 0.0)
    assert r_steps > 0  # the artificial stress was exercised
    st = ctx.status()
    assert st["error_flags"] == 0 and st["out_of_grid"] == 0
    vel = ctx.get("vel")
    if kind == "rings":
        # the rings have met: the velocity of some particles has changed, and the total
        # momentum (zero at the start: as many particles at +200 as at -200) has stayed zero
        assert np.abs(np.abs(vel[:, 0]) - 200.0).max() > 1.0
        assert abs(vel[:, 0].sum()) <= 1e-9 * np.abs(vel[:, 0]).sum()
    else:
        # the disc has reached the wall: some wall particles move; the fixed rows do not
        fixed = ctx.get("fixed") == 1.0
        wall = ctx.get("pos")[:, 0] > -0.01
        assert np.abs(vel[wall & ~fixed]).max() > 0.0
        assert np.all(vel[fixed] == 0.0)


@pytest.mark.parametrize("kind,nbox,grid_kind", [("rings", 21, 0), ("impact", 17, 0), ("impact", 17, 1)])
def test_mixed_form_rates_on_validation_scenes(mf, kind, nbox, grid_kind):
    """The mixed form (FP32 pair sums on cell-relative coordinates) on the SI-unit scenes and
    the adaptive grid: one step's rates against the FP64 form's from the same state, after a few
    FP64 steps so that the rings touch and the disc's support reaches the wall (norm-wise 1e-4,
    as on the cut)."""
    sc = getattr(mf.Scene, kind)(nbox)
    a = mf.Context(0)
    a.upload_scene(sc, grid_kind)
    a.step(5)
    b = mf.Context(0)
    b.upload_scene(sc, grid_kind)
    for f in LOADED:
        b.set(f, a.get(f))
    b.set_options(mf.THERMAL_BROOKSHAW, mf.JC_JOHNSON_COOK, mf.PRECISION_MIXED)
    for ctx in (a, b):
        for s in range(3):  # cell list, predictor, pair sums and rates
            ctx.stage(s)
    nb = a.get("blanked") == 0.0
    for f in RATES:
        x, y = b.get(f)[nb], a.get(f)[nb]
        assert np.isfinite(x).all(), f
        assert np.abs(y).max() > 0.0, f
        assert rel_err(x, y) < 1e-4, (f, rel_err(x, y))
