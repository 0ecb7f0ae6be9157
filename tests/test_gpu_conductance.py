"""Tool-workpiece contact conductance (mf_set_contact_conductance), an extension the benchmark
configuration at ~150k particles names (1e8 W/m^2K, tool at 300 K) and the reference does not
have: its heat crosses the interface only through the sampled tool particles' conduction terms
(interactions_gpu.cu:314-326). Off by default, so every parity test runs the reference's step.

Checked against its definition, from one state, one step with and one without it: a workpiece
particle in contact (nonzero contact force) that does not yield gains exactly
dt h (T_tool - T) / (cp sqrt(m rho)), T and rho being the step's result without conductance;
every other particle, and every other field, is bit for bit the step without it."""
import numpy as np
import pytest

from helpers import load_product, perturbed_scene

pytestmark = pytest.mark.gpu

H_CONTACT = 1e-7  # 1e8 W/m^2K in g/(us^3 K)
T_TOOL = 600.0


@pytest.mark.parametrize("precision", [0, 1])
def test_conductance_increment_matches_its_definition(mf, precision):
    st = perturbed_scene(mf, ny=12, seed=41)
    on = load_product(mf, st, precision=precision)
    off = load_product(mf, st, precision=precision)
    on.set_contact_conductance(H_CONTACT, T_TOOL)
    on.step(1)
    off.step(1)
    for f in ("pos", "vel", "S", "rho", "fc", "ft", "idx", "blanked"):
        assert np.array_equal(on.get(f), off.get(f)), f
    T_on, T_off = on.get("T"), off.get("T")
    contact = (np.abs(off.get("fc")).sum(axis=1) > 0) & (off.get("tool_p") == 0.0) & (off.get("blanked") == 0.0)
    elastic = (off.get("eps_pl_dot") == 0.0) & (on.get("eps_pl_dot") == 0.0) & (off.get("fixed") == 0.0)
    sel = contact & elastic
    assert sel.sum() > 5
    s = st["trml_wp"]
    m = st["phys"].mass
    rho = off.get("rho")
    expect = T_off + st["dt"] * H_CONTACT * (T_TOOL - T_off) / (s.cp * np.sqrt(m * rho))
    inc = T_on[sel] - T_off[sel]
    assert np.all(inc > 0)  # the tool is hotter
    assert np.allclose(T_on[sel], expect[sel], rtol=1e-13, atol=0.0)
    assert np.array_equal(T_on[~contact], T_off[~contact])
    on.close()
    off.close()
    # h = 0 is the reference's step, bit for bit
    zero = load_product(mf, st, precision=precision)
    ref = load_product(mf, st, precision=precision)
    zero.set_contact_conductance(0.0, T_TOOL)
    zero.step(2)
    ref.step(2)
    for f in ("pos", "vel", "S", "rho", "T", "eps_pl", "fc", "ft"):
        assert np.array_equal(zero.get(f), ref.get(f)), f
    zero.close()
    ref.close()


def test_conductance_refusals(mf):
    st = perturbed_scene(mf, ny=8, seed=42)
    c = load_product(mf, st)
    for bad in ((-1e-7, 300.0), (float("nan"), 300.0), (1e-7, float("inf"))):
        with pytest.raises(mf.MfError):
            c.set_contact_conductance(*bad)
    c.set_contact_conductance(H_CONTACT, 300.0)
    with pytest.raises(mf.MfError):  # no differentiable step with it
        c.tangent_mean_force(0, 2, 0)
    b = mf.Batch([c], steps_per_launch=2)
    assert not b.fused  # the child-graph batch runs the context's own step
    b.close()
    c.close()
