"""One leap-frog step on the GPU against the oracle, stage by stage and end to end.

Tolerances (norm-wise, max|a-b| / max|b| per field):
  * predictor outputs: 1e-13 (FMA contraction in the device code, none in the oracle);
  * artificial stress R: 1e-5 (the reference's atan2f/cosf/sinf in float: CUDA's device
    versions and glibc's differ by a few float ulps);
  * pair sums / rates given identical inputs: 1e-12;
  * corrector .. contact given identical inputs: 1e-12;
  * full steps with compressive states (R = 0): 1e-11;
  * eps_pl_dot: 1e-7, because the reference rounds the plastic multiplier to float
    (fmaxf, actions_gpu.cu:264-265): a last-bit difference of the secant result between
    CUDA's and glibc's pow/log moves it by one float ulp.
Cell lists, flags, permutations and the tool are compared bit for bit.
"""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import bits_equal, rel_err
from helpers import load_oracle, load_product, perturbed_scene

pytestmark = pytest.mark.gpu

STATE = ("pos", "vel", "S", "rho", "T", "eps_pl", "eps_pl_dot", "fc", "ft", "n")
RATES = ("pos_t", "vel_t", "S_t", "rho_t", "T_t")


FLOAT_ROUNDED = {"eps_pl_dot": 1e-7}


def check(ctx, o, fields, tol, mask=None):
    worst = {}
    for f in fields:
        ftol = max(tol, FLOAT_ROUNDED.get(f, 0.0))
        a, b = ctx.get(f), o.get(f)
        if mask is not None:
            a, b = a[mask], b[mask]
        e = rel_err(a, b)
        worst[f] = e
        assert np.isfinite(a).all() == np.isfinite(b).all(), f
        assert e <= ftol, (f, e)
    return worst


def tool_bits(mf, orc, ctx, o):
    t = mf.tool_to_array(ctx.tool_get())
    ot = o.get_tool()
    pt = mf.ToolState()
    C.memmove(C.byref(pt), C.byref(ot), C.sizeof(mf.ToolState))
    u = mf.tool_to_array(pt)
    return bits_equal(t["seg"], u["seg"]) and bits_equal(t["fillet"], u["fillet"])


@pytest.mark.parametrize("thermal_solver", [0, 1])
@pytest.mark.parametrize("tensile", [False, True])
def test_stages_against_oracle(mf, orc, thermal_solver, tensile):
    st = perturbed_scene(mf, ny=12, seed=11, tensile=tensile)
    ctx = load_product(mf, st, thermal_solver=thermal_solver, flags=mf.OPT_KEEP_DERIVATIVES)
    o = load_oracle(orc, st, thermal_solver=thermal_solver)
    # stage 0+1: sort, predictor, EOS, artificial stress
    ctx.stage(0)
    ctx.stage(1)
    o.L.orc_grid_update(o.s)
    o.L.orc_stage_predict(o.s)
    assert np.array_equal(ctx.get("hash"), o.get("hash"))
    assert np.array_equal(ctx.get("idx"), o.get("idx"))
    check(ctx, o, ("pos", "vel", "S", "rho", "T"), 1e-13)
    check(ctx, o, ("p",), 1e-14)
    eR = rel_err(ctx.get("R"), o.get("R"))
    assert eR <= 1e-5
    if not tensile:
        assert np.all(ctx.get("R") == 0.0) and np.all(o.get("R") == 0.0)
    # stage 2 with identical inputs: pair sums and rates
    o.set_field("R", ctx.get("R"))
    ctx.stage(2)
    o.L.orc_stage_interact(o.s)
    o.L.orc_stage_rates(o.s)
    wp = ctx.get("tool_p") == 0.0
    nb = ctx.get("blanked") == 0.0
    check(ctx, o, ("S_der", "v_der"), 1e-12, mask=wp & nb)
    check(ctx, o, RATES, 1e-12, mask=nb)
    # stage 3 with identical inputs: corrector .. invalidate
    for f in RATES:
        o.set_field(f, ctx.get(f))
    ctx.stage(3)
    o.L.orc_stage_finish(o.s)
    check(ctx, o, STATE, 1e-12)
    assert np.array_equal(ctx.get("blanked"), o.get("blanked"))
    assert tool_bits(mf, orc, ctx, o)
    # contact is really exercised by this state
    assert np.count_nonzero(np.abs(o.get("fc")).sum(axis=1)) > 5


@pytest.mark.parametrize("grid_kind", [0, 1])
def test_full_steps_compressive(mf, orc, grid_kind):
    st = perturbed_scene(mf, ny=12, seed=12, tensile=False)
    ctx = load_product(mf, st, grid_kind=grid_kind)
    o = load_oracle(orc, st, grid_kind=grid_kind)
    for k in range(5):
        ctx.step(1)
        o.L.orc_step(o.s)
        assert np.array_equal(ctx.get("idx"), o.get("idx")), k
        if np.any(ctx.get("R") != 0) or np.any(o.get("R") != 0):
            tol = 1e-6
        else:
            tol = 1e-11
        check(ctx, o, STATE + RATES, tol)
        assert np.array_equal(ctx.get("blanked"), o.get("blanked"))
    assert tool_bits(mf, orc, ctx, o)
    # the persistent particle number: a permutation, equal to the Rothlin grid's own id
    pid = ctx.get("id")
    assert np.array_equal(np.sort(pid), np.arange(st["N"]))
    if grid_kind == 1:
        assert np.array_equal(pid, ctx.get("idx"))
    # per-particle forces matched above; the net force cancels, so check the reduction
    # itself: the compensated device sum against the exact sum of the device's own forces
    f1 = ctx.report_force()
    fc, ft = ctx.get("fc"), ctx.get("ft")
    exact = np.array([math.fsum(np.concatenate([fc[:, k], ft[:, k]])) for k in range(2)])
    scale = np.abs(fc).sum(axis=0) + np.abs(ft).sum(axis=0)
    assert np.all(np.abs(f1 - exact) <= 1e-15 * scale)
    assert rel_err(f1, o.report_force()) <= 1e-8


def test_graphs_match_direct_launches(mf):
    st = perturbed_scene(mf, ny=10, seed=13, tensile=True)
    a = load_product(mf, st)
    b = load_product(mf, st, flags=mf.OPT_NO_GRAPHS)
    a.step(7)
    b.step(7)
    for f in STATE + RATES + ("idx", "hash", "blanked"):
        assert bits_equal(a.get(f), b.get(f)) if f not in ("idx", "hash") else np.array_equal(a.get(f), b.get(f)), f
    assert bits_equal(a.force_log(), b.force_log())


def test_deterministic(mf):
    st = perturbed_scene(mf, ny=10, seed=14, tensile=True)
    a = load_product(mf, st)
    b = load_product(mf, st)
    a.step(10)
    b.step(10)
    for f in STATE + RATES:
        assert bits_equal(a.get(f), b.get(f)), f


def test_blanked_particles_and_nan_cascade(mf, orc):
    """NaN in one particle's stress: the reference multiplies it by W = 0 for every window
    candidate, so its whole 5x5 window turns NaN and is blanked one step later."""
    st = perturbed_scene(mf, ny=12, seed=15, blank_frac=0.02)
    wp = np.flatnonzero(st["tool_p"] == 0.0)
    st["S"][wp[len(wp) // 2]] = np.nan
    ctx = load_product(mf, st)
    o = load_oracle(orc, st)
    for _ in range(3):
        ctx.step(1)
        o.L.orc_step(o.s)
        assert np.array_equal(ctx.get("blanked"), o.get("blanked"))
    nb = ctx.get("blanked") == 0.0
    assert (~nb).sum() > 0.02 * st["N"] + 5
    # the NaN stress also ran the secant solve to its cap (plasticity.cuh:112-115)
    assert ctx.status()["secant_cap_hits"] > 0
    check(ctx, o, ("pos", "vel", "rho"), 1e-9, mask=nb)


@pytest.mark.parametrize("jc_model", [0, 1])
def test_return_map_over_the_yield_surface(mf, orc, jc_model):
    """Many particles over the yield surface, Johnson-Cook (the four-lane solve) and the tanh
    law (the one-lane solve): one finish stage against the oracle."""
    st = perturbed_scene(mf, ny=10, seed=16, tensile=True)
    st["S"] *= 3.0  # push particles over the yield surface
    ctx = load_product(mf, st, jc_model=jc_model)
    o = load_oracle(orc, st, jc_model=jc_model)
    ctx.stage(0)
    ctx.stage(1)
    o.L.orc_grid_update(o.s)
    o.L.orc_stage_predict(o.s)
    o.set_field("R", ctx.get("R"))
    ctx.stage(2)
    o.L.orc_stage_interact(o.s)
    o.L.orc_stage_rates(o.s)
    for f in RATES:
        o.set_field(f, ctx.get(f))
    ctx.stage(3)
    o.L.orc_stage_finish(o.s)
    check(ctx, o, STATE, 1e-12)
    assert np.count_nonzero(ctx.get("eps_pl_dot")) > 10


def test_report_force_and_log(mf, orc):
    st = perturbed_scene(mf, ny=12, seed=17)
    ctx = load_product(mf, st)
    o = load_oracle(orc, st)
    forces = []
    for _ in range(4):
        ctx.step(1)
        o.L.orc_step(o.s)
        forces.append(o.report_force())
    log = ctx.force_log()
    assert log.shape == (4, 2)
    assert rel_err(log, np.array(forces)) <= 1e-9
    assert rel_err(ctx.report_force(), forces[-1]) <= 1e-9
    assert np.abs(forces[-1]).max() > 0


def test_host_writes_and_stages_between_steps(mf, orc):
    """With a locked grid each step's finish kernel already hashes and counts the particles
    for the next step. A host write of the state, or a staged step, in between must discard
    those counts: the steps after it still match the oracle."""
    st = perturbed_scene(mf, ny=12, seed=18, tensile=False)
    ctx = load_product(mf, st)
    o = load_oracle(orc, st)

    def steps(n, tol):
        ctx.step(n)
        for _ in range(n):
            o.L.orc_step(o.s)
        # stale counts would show here first: the cell lists are compared bit for bit
        assert np.array_equal(ctx.get("idx"), o.get("idx"))
        assert np.array_equal(ctx.get("hash"), o.get("hash"))
        if np.any(ctx.get("R") != 0) or np.any(o.get("R") != 0):
            tol = 1e-6  # artificial stress active: float-narrowed atan2f/cosf/sinf
        check(ctx, o, STATE + RATES, tol)
        assert tool_bits(mf, orc, ctx, o)

    steps(3, 1e-11)
    # move particles across cell borders from the host: the prepared counts are stale.
    # The displaced particles form close pairs whose large pair forces amplify the
    # last-bit differences of FMA contraction, hence the wider tolerance afterwards.
    pos = ctx.get("pos")
    wp = np.flatnonzero(ctx.get("tool_p") == 0.0)
    rng = np.random.default_rng(5)
    sel = rng.choice(wp, size=len(wp) // 10, replace=False)
    pos[sel] += rng.uniform(-0.6, 0.6, (len(sel), 2)) * (st["grid"][2] / 1.5)
    ctx.set("pos", pos)
    o.set_field("pos", pos)
    steps(2, 1e-9)
    # one staged step, then graph steps again
    for k in range(4):
        ctx.stage(k)
    o.L.orc_step(o.s)
    steps(3, 1e-9)
