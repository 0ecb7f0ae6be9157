"""The reference's validation scenes run through the oracle on the CPU (the checker the GPU
parity tests of these scenes compare against): physical properties that hold whatever the
resolution.

  * rings (setup_rings, benchmarks.cpp:161-253): equal numbers of particles at +200 and -200 and
    pair forces that cancel pairwise (the same h everywhere, no tool, nothing fixed), so the
    total momentum stays zero while the rings collide and slow down;
  * impact (setup_impact, benchmarks.cpp:23-159): the disc reaches the wall within the first
    steps (its kernel support already overlaps the wall), the wall's fixed rows stay at rest,
    the contact zone yields (Johnson-Cook, steel at 1000 m/s).
"""
import ctypes as C

import numpy as np
import pytest


def oracle_scene(mf, orc, sc, grid_kind=0):
    s = sc.s
    o = orc.Oracle(sc.N)
    for k in ("pos", "vel", "rho", "T", "h", "fixed", "tool_p"):
        o.set_field(k, sc.array(k))
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


def test_rings_collide_with_zero_total_momentum(mf, orc):
    sc = mf.Scene.rings(21)
    o = oracle_scene(mf, orc, sc)
    v0 = o.get("vel")
    assert v0[:, 0].sum() == 0.0 and np.all(np.abs(v0[:, 0]) == 200.0)
    assert o.L.orc_steps(o.s, 20) == 0
    vel = o.get("vel")
    assert np.isfinite(vel).all() and o.get("blanked").sum() == 0
    assert np.abs(np.abs(vel[:, 0]) - 200.0).max() > 10.0  # the rings have met
    assert abs(vel[:, 0].sum()) <= 1e-12 * np.abs(vel[:, 0]).sum()
    assert abs(vel[:, 1].sum()) <= 1e-12 * np.abs(vel[:, 0]).sum()
    assert np.all(o.get("eps_pl") == 0.0)  # no plasticity in this scene


@pytest.mark.parametrize("grid_kind", [0, 1])
def test_impact_yields_and_holds_the_fixed_rows(mf, orc, grid_kind):
    sc = mf.Scene.impact(17)
    o = oracle_scene(mf, orc, sc, grid_kind)
    assert o.L.orc_steps(o.s, 12) == 0
    vel, pos = o.get("vel"), o.get("pos")
    fixed = o.get("fixed") == 1.0
    wall = pos[:, 0] > -0.01
    assert np.isfinite(vel).all() and o.get("blanked").sum() == 0
    assert np.all(vel[fixed] == 0.0)
    assert np.abs(vel[wall & ~fixed]).max() > 10.0
    assert (o.get("eps_pl") > 0.0).sum() > 10
    assert o.L.orc_out_of_grid(o.s) == 0
