"""The oracle against the golden vectors of the reference's own sources (CPU only).

The fixtures in tests/golden/ come from the reference's kernels.cuh, plasticity.cuh,
tool.cpp and geometric_primitives.cpp compiled on the host (tests/golden/make_golden.py).
The oracle must reproduce them bit for bit: same expressions, same order, same libm.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import bits_equal


def test_cubic_spline_and_pse_bitwise(orc, golden):
    g = golden("ref_kernels")
    L = orc.lib()
    o = np.zeros(3)
    w = np.zeros_like(g["w"])
    pse = np.zeros_like(g["pse"])
    for i in range(g["h"].size):
        L.orc_cubic_spline(g["xi"][i], g["yi"][i], g["xj"][i], g["yj"][i], g["h"][i], o.ctypes.data_as(C.c_void_p))
        w[i] = o
        pse[i] = L.orc_lapl_pse(g["xi"][i], g["yi"][i], g["xj"][i], g["yj"][i], g["h"][i])
    assert bits_equal(w, g["w"])
    assert bits_equal(pse, g["pse"])
    # the r^2 < 1e-8 cut (kernels.cuh:43) is part of the fixture
    assert np.all(g["w"][20:40] == 0.0)


def test_johnson_cook_and_secant_bitwise(orc, golden):
    g = golden("ref_plasticity")
    L = orc.lib()
    J = orc.joco_struct(g["jc"])
    n = g["eps"].size
    sy = np.array([L.orc_sigma_yield(C.byref(J), g["eps"][i], g["epsdot"][i], g["T"][i]) for i in range(n)])
    syt = np.array([L.orc_sigma_yield_tanh(C.byref(J), g["eps"][i], g["epsdot"][i], g["T"][i]) for i in range(n)])
    assert bits_equal(sy, g["sigma_yield"])
    assert bits_equal(syt, g["sigma_yield_tanh"])
    mu = float(g["mu"])
    for model, key in ((0, "secant_jc"), (1, "secant_tanh")):
        sec = np.array([L.orc_solve_secant(C.byref(J), model, g["init"][i], 1e-6, g["norm"][i], g["eps"][i], g["T"][i],
                                           g["dt"][i], mu, None) for i in range(n)])
        assert bits_equal(sec, g[key]), key


def test_tool_lines_after_translation(orc, golden):
    """tool::update_tool (tool.cpp:211-221) = 50 translations + line(left, right)."""
    g = golden("ref_tools")
    L = orc.lib()
    k = 0
    while f"t{k}_seg" in g:
        seg = g[f"t{k}_seg"].copy()
        for _ in range(50):
            seg[:, 0] = seg[:, 0] + 1.17e-3 * 1.16667e-4
            seg[:, 1] = seg[:, 1] + 1.17e-3 * 0.0
            seg[:, 2] = seg[:, 2] + 1.17e-3 * 1.16667e-4
            seg[:, 3] = seg[:, 3] + 1.17e-3 * 0.0
        a, b, v = C.c_double(), C.c_double(), C.c_int()
        for s in seg:
            L.orc_line_from_points(s[0], s[1], s[2], s[3], C.byref(a), C.byref(b), C.byref(v))
            s[4], s[5], s[6] = a.value, b.value, float(v.value)
        assert bits_equal(seg, g[f"t{k}_seg_moved"]), k
        k += 1
    assert k == 4


def test_live_reference_randomised(orc):
    """Fresh random cases against the host-compiled reference, where it was built."""
    R = orc.ref()
    if R is None:
        pytest.skip("reference sources not built here (fixtures cover this case)")
    L = orc.lib()
    rng = np.random.default_rng(7)
    o1, o2 = np.zeros(3), np.zeros(3)
    for _ in range(3000):
        h = rng.uniform(1e-5, 1e-1)
        xi, yi = rng.uniform(-1, 1, 2)
        r = h * rng.uniform(0, 2.1)
        a = rng.uniform(0, 2 * np.pi)
        args = (xi, yi, xi + r * np.cos(a), yi + r * np.sin(a), h)
        L.orc_cubic_spline(*args, o1.ctypes.data_as(C.c_void_p))
        R.refh_cubic_spline(*args, o2.ctypes.data_as(C.c_void_p))
        assert bits_equal(o1, o2)


def test_usui_wear_bitwise(orc, golden):
    """Usui wear rate (tool_wear.cu:20-64): the oracle against the reference's own eval_usui."""
    g = golden("ref_usui")
    n = len(g["h"])
    o = orc.Oracle(n)
    for k in ("pos", "vel", "fc", "ft", "h", "n", "T"):
        o.set_field(k, g[k])
    out = o.usui(float(g["K"]), float(g["alpha"]), g["tool_vel"])
    assert bits_equal(out, g["usui"][:3])
    assert bits_equal(float(g["dt"]) * out[2], g["usui"][3])  # m_accum_wear += dt * avg


@pytest.mark.parametrize("thermal_solver,jc_model", [(0, 0), (1, 0), (0, 1)])
def test_oracle_on_the_reference_functions_is_the_same_bit_for_bit(mf, orc, thermal_solver, jc_model):
    """The oracle stepping with the reference's own host-compiled kernels.cuh / plasticity.cuh
    functions at their call sites (the CPU baseline's reference form) equals the restatement
    bit for bit: three steps of a cut with contact, yielding and heat conduction (with the tanh
    yield law the return map keeps the restatement; the kernels are still the reference's)."""
    if orc.ref() is None:
        pytest.skip("the reference's sources were not built here")
    from helpers import load_oracle, perturbed_scene
    st = perturbed_scene(mf, ny=10, seed=71, tensile=True)
    st["S"] *= 3.0  # particles over the yield surface
    a = load_oracle(orc, st, thermal_solver=thermal_solver, jc_model=jc_model)
    b = load_oracle(orc, st, thermal_solver=thermal_solver, jc_model=jc_model)
    assert orc.use_reference_functions(b)
    for _ in range(3):
        assert a.L.orc_step(a.s) == 0 and b.L.orc_step(b.s) == 0
    for f in ("pos", "vel", "S", "rho", "T", "eps_pl", "eps_pl_dot", "fc", "ft", "pos_t", "vel_t", "S_t", "rho_t",
              "T_t", "blanked"):
        assert bits_equal(a.get(f), b.get(f)), f
    assert (a.get("eps_pl") > 0.0).sum() > 10  # the return map ran


def test_oracle_step_fixtures(mf, orc, golden):
    """The oracle's own step on the benchmark configurations against its fixtures: c1 after one
    step (arrays, bit for bit) and 1,000 steps, c2 after one step (digests of every per-particle
    field). A regression pin of the checker itself (tests/golden/oracle_steps.py)."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import oracle_steps

    g = golden("oracle_steps")
    o = oracle_steps.run(mf, orc, "c1", 1)
    for f in oracle_steps.ARRAY_FIELDS:
        assert bits_equal(o.get(f), g["c1_step1_" + f]), f
    assert oracle_steps.digest(o) == str(g["c1_step1_sha256"])
    assert oracle_steps.digest(oracle_steps.run(mf, orc, "c1", 1000)) == str(g["c1_step1000_sha256"])
    assert oracle_steps.digest(oracle_steps.run(mf, orc, "c2", 1)) == str(g["c2_step1_sha256"])
