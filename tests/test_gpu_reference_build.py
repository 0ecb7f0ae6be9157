"""The reference's own FP64 CUDA build (oracle/_ref/libref_gpu.so: its device sources compiled
unchanged for sm_100a, with a shim for the texture-reference API that CUDA 12 removed) as the
GPU oracle, next to the CPU restatement.

  * the CPU oracle against the reference build, full steps of a compressive state (R = 0, so
    the float trigonometry of the artificial stress, where glibc and CUDA differ by a few float
    ulps, does not enter): this pins the oracle's step bodies (pair loop, actions, contact,
    sort) to the reference's own kernels;
  * the product's FP64 step against the reference build on the same GPU: compressive and
    tensile states (both sides use CUDA's atan2f/cosf/sinf, so R is compared too), and the
    ~150k-particle benchmark cut from its initial state.

R is compared on workpiece particles only: the reference leaves a tool particle's R (an array
indexed by position, which the sort does not move) at whatever an earlier occupant of that
position left there, and never reads it. Tolerances, norm-wise max|a-b| / max|b| per field: rates 1e-12 and state 1e-11 over five steps
(FMA contraction patterns and the reference's thrust reduction order differ); eps_pl_dot 1e-7
(the reference rounds the plastic multiplier to float, so a last-bit difference of its input
moves it by a float ulp); the tool force within 1e-9 of the total contact force magnitude
(thrust::reduce sums in an unspecified order). Cell lists, blanking and the tool bit for bit.

The reference keeps its constants and option flags process-wide, so every reference system
here uses the same options: Johnson-Cook plasticity, heat, friction heat and a tool. Its heat
solver is chosen at compile time (types.h): the default build runs Brookshaw, a second build
(oracle/_ref/libref_gpu_pse.so, the switch turned in a generated copy of types.h) its PSE
solver, which pins the product's PSE path on a perturbed scene and on the ~500k-particle
configuration.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import bits_equal, rel_err
from helpers import load_oracle, load_product, perturbed_scene, scene_state

pytestmark = pytest.mark.gpu

STATE = ("pos", "vel", "S", "rho", "T", "eps_pl", "eps_pl_dot", "fc", "ft", "n")
RATES = ("pos_t", "vel_t", "S_t", "rho_t", "T_t")
EXTRA = ("S", "eps_pl", "eps_pl_dot", "fc", "ft", "n", "pos_t", "vel_t", "rho_t", "S_t", "T_t", "blanked")
FLOAT_ROUNDED = {"eps_pl_dot": 1e-7}


def _doubles(struct):
    return [getattr(struct, f) for f, _ in struct._fields_]


def ref_gpu_from(orc, st, solver="brookshaw"):
    if orc.ref_gpu(solver) is None:
        pytest.skip("the reference's GPU build was not made (no reference tree where the build ran)")
    tool = orc.OrcTool()
    C.memmove(C.byref(tool), C.byref(st["tool"]), C.sizeof(orc.OrcTool))
    r = orc.RefGPU(st, _doubles(st["phys"]), _doubles(st["corr"]), _doubles(st["joco"]), _doubles(st["trml_wp"]),
                   _doubles(st["trml_tool"]), tool, solver=solver)
    for k in EXTRA:
        r.set_field(k, st[k])
    return r


def compare(a_get, b_get, fields, tol, mask=None):
    worst = {}
    for f in fields:
        a, b = a_get(f), b_get(f)
        if mask is not None:
            a, b = a[mask], b[mask]
        assert np.isfinite(a).all() == np.isfinite(b).all(), f
        e = rel_err(a, b)
        worst[f] = e
        assert e <= max(tol, FLOAT_ROUNDED.get(f, 0.0)), (f, e)
    return worst


def tool_bits(mf, a, b):
    ta, tb = mf.ToolState(), mf.ToolState()
    C.memmove(C.byref(ta), C.byref(a), C.sizeof(mf.ToolState))
    C.memmove(C.byref(tb), C.byref(b), C.sizeof(mf.ToolState))
    u, v = mf.tool_to_array(ta), mf.tool_to_array(tb)
    return bits_equal(u["seg"], v["seg"]) and bits_equal(u["fillet"], v["fillet"])


def force_close(F, Fr, fc, ft):
    total = np.abs(fc).sum() + np.abs(ft).sum()
    return bool(np.all(np.abs(F - Fr) <= 1e-9 * max(total, 1e-300)))


def test_oracle_against_reference_build_compressive(mf, orc):
    """Full steps of a compressive state with contact and friction: the CPU oracle's step equals
    the reference's own CUDA step for as long as the artificial stress stays zero on both sides
    (at least two steps; tension, and with it R, appears after a few steps)."""
    st = perturbed_scene(mf, ny=12, seed=31, tensile=False)
    o = load_oracle(orc, st)
    r = ref_gpu_from(orc, st)
    compared = 0
    for k in range(5):
        o.L.orc_step(o.s)
        r.step(1)
        wp = r.get("tool_p") == 0.0  # tool particles' R is stale in the reference, unread
        if not (np.all(o.get("R")[wp] == 0.0) and np.all(r.get("R")[wp] == 0.0)):
            break
        assert np.array_equal(o.get("idx"), r.get("idx")), k
        assert np.array_equal(o.get("hash"), r.get("hash")), k
        assert np.array_equal(o.get("blanked"), r.get("blanked")), k
        compare(o.get, r.get, RATES, 1e-12)
        compare(o.get, r.get, STATE, 1e-11)
        assert force_close(o.report_force(), r.report_force(), r.get("fc"), r.get("ft")), k
        assert tool_bits(mf, o.get_tool(), r.get_tool())
        assert np.count_nonzero(np.abs(r.get("fc")).sum(axis=1)) > 5
        compared += 1
    assert compared >= 2


@pytest.mark.parametrize("tensile", [False, True])
def test_product_against_reference_build(mf, orc, tensile):
    """Five steps of the product's FP64 form against the reference's own CUDA step, same GPU."""
    st = perturbed_scene(mf, ny=12, seed=32, tensile=tensile)
    ctx = load_product(mf, st)
    r = ref_gpu_from(orc, st)
    r_nonzero = 0
    for k in range(5):
        ctx.step(1)
        r.step(1)
        assert np.array_equal(ctx.get("idx"), r.get("idx")), k
        assert np.array_equal(ctx.get("hash"), r.get("hash")), k
        assert np.array_equal(ctx.get("blanked"), r.get("blanked")), k
        nb = r.get("blanked") == 0.0
        wp = nb & (r.get("tool_p") == 0.0)  # tool particles' R is stale in the reference, unread
        r_nonzero += int(np.any(r.get("R")[wp] != 0.0))
        compare(ctx.get, r.get, ("R",), 1e-12, wp)
        compare(ctx.get, r.get, RATES, 1e-12, nb)
        compare(ctx.get, r.get, STATE, 1e-11, nb)
        assert force_close(ctx.report_force(), r.report_force(), r.get("fc"), r.get("ft")), k
        start, end = ctx.cells()
        rs, re = r.cells()
        assert np.array_equal(start, rs), k
        occ = rs != -1
        assert np.array_equal(end[occ], re[occ]), k
    if tensile:
        assert r_nonzero > 0  # the artificial stress was exercised (both sides' CUDA float trigonometry)
    pt = orc.OrcTool()
    t = ctx.tool_get()
    C.memmove(C.byref(pt), C.byref(t), C.sizeof(orc.OrcTool))
    assert tool_bits(mf, pt, r.get_tool())
    ctx.close()


def test_product_against_reference_build_benchmark_cut(mf, orc):
    """The ~150k-particle cut (176,695 particles, Brookshaw, sampled tool) from its initial
    state: five steps of the product's FP64 form against the reference's own CUDA step."""
    import bench

    p, solver, _ = bench.config_params(mf, "c2")
    sc = mf.Scene.from_params(p)
    st = scene_state(mf, sc)
    ctx = load_product(mf, st, thermal_solver=solver)
    r = ref_gpu_from(orc, st)
    for k in range(5):
        ctx.step(1)
        r.step(1)
        assert np.array_equal(ctx.get("idx"), r.get("idx")), k
        assert np.array_equal(ctx.get("blanked"), r.get("blanked")), k
        nb = r.get("blanked") == 0.0
        wp = nb & (r.get("tool_p") == 0.0)
        compare(ctx.get, r.get, ("R",), 1e-12, wp)
        compare(ctx.get, r.get, RATES, 1e-12, nb)
        compare(ctx.get, r.get, STATE, 1e-11, nb)
        assert force_close(ctx.report_force(), r.report_force(), r.get("fc"), r.get("ft")), k
    ctx.close()


def test_product_against_reference_build_mid_cut(mf, orc, c2_midcut):
    """The same cut after 0.05 mm of the product's FP64 cut (contact, friction, friction heat
    and yielding active), loaded into the reference build: five steps of each."""
    sc, solver = c2_midcut["scene"], c2_midcut["solver"]
    ctx = mf.Context(0)
    ctx.upload_scene(sc, mf.GRID_GREEN)
    ctx.set_options(solver, mf.JC_JOHNSON_COOK, mf.PRECISION_FP64)
    ctx.state_load(str(c2_midcut["path"]))
    st = scene_state(mf, sc)
    for k in ("pos", "vel", "rho", "T", "h", "fixed", "tool_p") + EXTRA:
        st[k] = ctx.get(k)
    st["tool"] = ctx.tool_get()
    r = ref_gpu_from(orc, st)
    plastic = 0
    for k in range(5):
        ctx.step(1)
        r.step(1)
        assert np.array_equal(ctx.get("idx"), r.get("idx")), k
        assert np.array_equal(ctx.get("blanked"), r.get("blanked")), k
        nb = r.get("blanked") == 0.0
        wp = nb & (r.get("tool_p") == 0.0)
        compare(ctx.get, r.get, ("R",), 1e-12, wp)
        compare(ctx.get, r.get, RATES, 1e-12, nb)
        compare(ctx.get, r.get, STATE, 1e-11, nb)
        assert force_close(ctx.report_force(), r.report_force(), r.get("fc"), r.get("ft")), k
        plastic = max(plastic, int(np.count_nonzero(r.get("eps_pl_dot")[nb])))
    assert np.count_nonzero(np.abs(r.get("fc")).sum(axis=1)) >= 10
    assert plastic >= 10
    ctx.close()


def product_steps_against(orc, ctx, r, steps):
    """`steps` full steps of both, compared after each (as in the Brookshaw tests above)."""
    for k in range(steps):
        ctx.step(1)
        r.step(1)
        assert np.array_equal(ctx.get("idx"), r.get("idx")), k
        assert np.array_equal(ctx.get("hash"), r.get("hash")), k
        assert np.array_equal(ctx.get("blanked"), r.get("blanked")), k
        nb = r.get("blanked") == 0.0
        wp = nb & (r.get("tool_p") == 0.0)
        compare(ctx.get, r.get, ("R",), 1e-12, wp)
        compare(ctx.get, r.get, RATES, 1e-12, nb)
        compare(ctx.get, r.get, STATE, 1e-11, nb)
        assert force_close(ctx.report_force(), r.report_force(), r.get("fc"), r.get("ft")), k
    pt = orc.OrcTool()  # the product's tool after the steps, for the bitwise tool check
    t = ctx.tool_get()
    C.memmove(C.byref(pt), C.byref(t), C.sizeof(orc.OrcTool))
    return pt


@pytest.mark.parametrize("tensile", [False, True])
def test_product_against_reference_pse_build(mf, orc, tensile):
    """The PSE heat solver (interactions_gpu.cu:88-144, leap_frog.cu:122): five steps of the
    product's FP64 form against the reference's own CUDA step built with its PSE solver, on the
    same GPU; heat flows (T_t nonzero) on both sides."""
    st = perturbed_scene(mf, ny=12, seed=34, tensile=tensile)
    ctx = load_product(mf, st, thermal_solver=mf.THERMAL_PSE)
    r = ref_gpu_from(orc, st, solver="pse")
    pt = product_steps_against(orc, ctx, r, 5)
    assert np.count_nonzero(r.get("T_t")) > 100
    assert tool_bits(mf, pt, r.get_tool())
    ctx.close()


def test_product_against_reference_pse_build_500k(mf, orc):
    """The ~500k-particle configuration (1290 x 387 lattice, dx = 1.55 um, 577,555 particles,
    PSE heat, where the half-length binding of tool_particle, interactions_gpu.cu:405, splits the
    particles at N/2): five steps of the product's FP64 form against the reference's PSE build."""
    import bench

    p, solver, _ = bench.config_params(mf, "c3")
    assert solver == mf.THERMAL_PSE
    sc = mf.Scene.from_params(p)
    st = scene_state(mf, sc)
    assert st["N"] > 500_000
    ctx = load_product(mf, st, thermal_solver=solver)
    r = ref_gpu_from(orc, st, solver="pse")
    pt = product_steps_against(orc, ctx, r, 5)
    assert tool_bits(mf, pt, r.get_tool())
    ctx.close()
