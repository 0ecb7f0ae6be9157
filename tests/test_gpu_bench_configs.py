"""The plain FP64 step against the oracle at the benchmark configurations' full sizes.

  * the ~150k-particle cut (714 x 214 lattice, dx = 2.8 um, + 23,899 sampled tool particles =
    176,695; Brookshaw heat; ~350k cells, ~690 finish-kernel chunks, the force reduction at
    full width), from its initial state and from a mid-cut state after 0.05 mm of FP64 cut,
    where contact, friction, friction heat and yielding are active;
  * the ~500k-particle cut (1290 x 387, dx = 1.55 um, 577,555 particles, PSE heat, whose
    half-length texture binding of tool_particle depends on N, interactions_gpu.cu:405).

Each runs five steps stage by stage, the oracle continuing from its own state. Compared per
step: the cell list (hash, permutation, cell bounds) bit for bit; the artificial stress R at
1e-5 (the reference's atan2f/cosf/sinf in float: CUDA's and glibc's differ by a few float
ulps), after which the oracle takes the product's R, as in the small-scene stage tests; rates
norm-wise 1e-12 on the first step from a common state and 1e-11 after it, state 1e-11
(eps_pl_dot 1e-7: the reference rounds the plastic multiplier to float); blanking and the tool
bit for bit; the tool force (report_force, output.cu:31-39)
within 1e-9 of the total contact force magnitude.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import bits_equal, rel_err

pytestmark = pytest.mark.gpu

LOADED = ("pos", "vel", "rho", "T", "h", "fixed", "tool_p", "S", "eps_pl", "eps_pl_dot", "fc", "ft", "n",
          "pos_t", "vel_t", "rho_t", "S_t", "T_t", "blanked")
STATE = ("pos", "vel", "S", "rho", "T", "eps_pl", "eps_pl_dot", "fc", "ft", "n")
RATES = ("pos_t", "vel_t", "S_t", "rho_t", "T_t")
FLOAT_ROUNDED = {"eps_pl_dot": 1e-7}


def config_scene(mf, name):
    import bench

    p, solver, _ = bench.config_params(mf, name)
    return mf.Scene.from_params(p), solver


def product(mf, sc, solver):
    ctx = mf.Context(0)
    ctx.upload_scene(sc, mf.GRID_GREEN)
    ctx.set_options(solver, mf.JC_JOHNSON_COOK, mf.PRECISION_FP64)
    return ctx


def oracle_from(orc, mf, ctx, sc, solver):
    """A fresh oracle holding the product's current state, tool, constants and grid."""
    s = sc.s
    o = orc.Oracle(sc.N)
    for k in LOADED:
        o.set_field(k, ctx.get(k))
    o.L.orc_set_grid_locked(o.s, 0, s.grid_bbmin[0], s.grid_bbmin[1], s.grid_bbmax[0], s.grid_bbmax[1], s.grid_h)
    phys = orc.OrcPhys(*[getattr(s.phys, f) for f, _ in orc.OrcPhys._fields_])
    corr = orc.OrcCorr(*[getattr(s.corr, f) for f, _ in orc.OrcCorr._fields_])
    joco = orc.OrcJoco(*[getattr(s.joco, f) for f, _ in orc.OrcJoco._fields_])
    tw = orc.OrcTrml(*[getattr(s.trml_wp, f) for f, _ in orc.OrcTrml._fields_])
    tt = orc.OrcTrml(*[getattr(s.trml_tool, f) for f, _ in orc.OrcTrml._fields_])
    o.L.orc_set_constants(o.s, C.byref(phys), C.byref(corr), C.byref(joco), C.byref(tw), C.byref(tt))
    o.L.orc_set_options(o.s, solver, 0)
    o.L.orc_set_dt(o.s, s.dt)
    tool = orc.OrcTool()
    t = ctx.tool_get()
    C.memmove(C.byref(tool), C.byref(t), C.sizeof(orc.OrcTool))
    o.L.orc_set_tool(o.s, C.byref(tool))
    o._keep = (phys, corr, joco, tw, tt, tool)
    return o


def compare(ctx, o, fields, tol, mask):
    for f in fields:
        a, b = ctx.get(f)[mask], o.get(f)[mask]
        assert np.isfinite(a).all() == np.isfinite(b).all(), f
        e = rel_err(a, b)
        assert e <= max(tol, FLOAT_ROUNDED.get(f, 0.0)), (f, e)


def tool_equal(mf, ctx, o):
    t = mf.tool_to_array(ctx.tool_get())
    pt = mf.ToolState()
    ot = o.get_tool()
    C.memmove(C.byref(pt), C.byref(ot), C.sizeof(mf.ToolState))
    u = mf.tool_to_array(pt)
    return bits_equal(t["seg"], u["seg"]) and bits_equal(t["fillet"], u["fillet"])


def staged_steps(mf, ctx, o, steps, first=True):
    """`steps` steps of both, stage by stage, compared after each; returns per-step counts of
    particles in contact and of particles that yielded (plastic strain rate > 0). The rates of
    the first step from a common state are compared at 1e-12; after that the two states have
    each been integrated on their own (only R is shared), and rates and state meet 1e-11."""
    contact, plastic = [], []
    for k in range(steps):
        ctx.stage(0)
        ctx.stage(1)
        assert o.L.orc_grid_update(o.s) == 0
        o.L.orc_stage_predict(o.s)
        assert np.array_equal(ctx.get("hash"), o.get("hash")), k
        assert np.array_equal(ctx.get("idx"), o.get("idx")), k
        a_start, a_end = ctx.cells()
        b_start, b_end = o.cells()
        assert np.array_equal(a_start, b_start), k
        occ = b_start != -1
        assert np.array_equal(a_end[occ], b_end[occ]), k
        R = ctx.get("R")
        assert rel_err(R, o.get("R")) <= 1e-5, k
        o.set_field("R", R)
        ctx.stage(2)
        o.L.orc_stage_interact(o.s)
        o.L.orc_stage_rates(o.s)
        ctx.stage(3)
        o.L.orc_stage_finish(o.s)
        blanked = ctx.get("blanked")
        assert np.array_equal(blanked, o.get("blanked")), k
        nb = blanked == 0.0
        compare(ctx, o, RATES, 1e-12 if (first and k == 0) else 1e-11, nb)
        compare(ctx, o, STATE, 1e-11, nb)
        assert tool_equal(mf, ctx, o), k
        fc, ft = o.get("fc"), o.get("ft")
        total = np.abs(fc).sum() + np.abs(ft).sum()
        F, Fo = ctx.report_force(), o.report_force()
        assert np.all(np.abs(F - Fo) <= 1e-9 * max(total, 1e-300)), (k, F, Fo)
        contact.append(int(np.count_nonzero(np.abs(fc).sum(axis=1))))
        plastic.append(int(np.count_nonzero(ctx.get("eps_pl_dot")[nb])))
    st = ctx.status()
    assert st["error_flags"] == 0 and st["out_of_grid"] == 0
    return contact, plastic


def test_c2_initial_state_five_steps(mf, orc):
    sc, solver = config_scene(mf, "c2")
    assert sc.N == 176_695
    ctx = product(mf, sc, solver)
    o = oracle_from(orc, mf, ctx, sc, solver)
    assert ctx.geometry()["num_cell"] > 300_000
    staged_steps(mf, ctx, o, 5)
    ctx.close()


def test_c2_mid_cut_five_steps(mf, orc, c2_midcut):
    """After 0.05 mm of FP64 cut (dt = 2.35e-4 us at 70 m/min: ~182k steps) the chip is
    forming: the five compared steps have particles in contact and yielding."""
    sc, solver = c2_midcut["scene"], c2_midcut["solver"]
    assert 150_000 < c2_midcut["steps"] < 220_000
    st = c2_midcut["status"]
    assert st["blanked"] == 0 and st["error_flags"] == 0 and st["out_of_grid"] == 0
    ctx = product(mf, sc, solver)
    ctx.state_load(str(c2_midcut["path"]))
    # the production step (one CUDA graph, fused hash) from this state, on a copy, must equal
    # the staged step that is compared with the oracle below
    twin = product(mf, sc, solver)
    twin.state_load(str(c2_midcut["path"]))
    twin.step(1)
    o = oracle_from(orc, mf, ctx, sc, solver)
    contact, plastic = staged_steps(mf, ctx, o, 1)
    assert np.array_equal(twin.get("idx"), ctx.get("idx"))
    for f in STATE + RATES:
        assert rel_err(twin.get(f), ctx.get(f)) <= 1e-14, f
    twin.close()
    c2, p2 = staged_steps(mf, ctx, o, 4, first=False)
    contact += c2
    plastic += p2
    assert min(contact) >= 10, contact
    assert min(plastic) >= 10, plastic
    ctx.close()


def test_c3_pse_initial_state_five_steps(mf, orc):
    sc, solver = config_scene(mf, "c3")
    assert solver == mf.THERMAL_PSE
    assert sc.N > 500_000
    ctx = product(mf, sc, solver)
    o = oracle_from(orc, mf, ctx, sc, solver)
    staged_steps(mf, ctx, o, 5)
    ctx.close()
