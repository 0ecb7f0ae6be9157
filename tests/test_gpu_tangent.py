"""The differentiable form: FP64 steps on dual numbers (mf_tangent_mean_force).

The objective is the window-averaged tool force (report_force per step, output.cu:31-39); the
parameters are Johnson-Cook A, B, n, C, m and the friction coefficient mu. The checks:
  * the dual run's values are the plain FP64 step's (same operations, same order);
  * each derivative agrees with FP64 central differences of the same objective within 1e-3
    relative. The central difference uses a relative step of 3e-3: the reference's return map
    rounds the plastic increment to float and takes float roots of doubles, which makes the
    objective a fine staircase, and at a relative step of 1e-4 that staircase still moves the
    difference quotients of the weakly coupled parameters (n, C, m) by ~1e-2;
  * the torch.autograd.Function wrapper returns the same derivatives.
"""
import importlib.util
import math
from pathlib import Path

import numpy as np
import pytest

from helpers import load_product, perturbed_scene

pytestmark = pytest.mark.gpu

WINDOW = 40
FD_REL_STEP = 3e-3


def autodiff_module():
    path = Path(__file__).resolve().parent.parent / "mfree_iwf-ul_cut_gpu_b200" / "autodiff.py"
    spec = importlib.util.spec_from_file_location("mfree_b200_autodiff", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def loaded_scene(mf):
    """Tool pushed into the workpiece, stresses tripled: contact, friction and yielding."""
    st = perturbed_scene(mf, ny=12, seed=21)
    st["S"] *= 3.0
    return st, load_product(mf, st)


def test_dual_values_are_the_fp64_step(mf):
    st, ctx = loaded_scene(mf)
    mean, dmean = ctx.tangent_mean_force(0, WINDOW, -1)
    assert np.all(dmean == 0.0)
    ref = load_product(mf, st)
    ref.step(WINDOW)
    log = ref.force_log()
    assert log.shape == (WINDOW, 2)
    np.testing.assert_allclose(mean, log.mean(axis=0), rtol=1e-12, atol=0.0)
    assert abs(mean[0]) > 0.0
    # the context's own state is left as it was
    assert np.array_equal(ctx.get("pos"), load_product(mf, st).get("pos"))


@pytest.mark.parametrize("param", range(6))
def test_derivative_against_central_differences(mf, param):
    ad = autodiff_module()
    st, ctx = loaded_scene(mf)
    theta0 = ad.current_parameters(ctx)
    _, d = ctx.tangent_mean_force(0, WINDOW, param)
    h = FD_REL_STEP * abs(theta0[param])
    th = list(theta0)
    th[param] += h
    ad.apply_parameters(ctx, th)
    fp, _ = ctx.tangent_mean_force(0, WINDOW, -1)
    th[param] -= 2 * h
    ad.apply_parameters(ctx, th)
    fm, _ = ctx.tangent_mean_force(0, WINDOW, -1)
    fd = (fp - fm) / (2 * h)
    assert np.all(np.abs(fd) > 0.0), ad.PARAMS[param]
    rel = np.abs(d - fd) / np.abs(fd)
    assert np.all(rel <= 1e-3), (ad.PARAMS[param], d, fd, rel)


def test_autograd_function(mf):
    torch = pytest.importorskip("torch")
    ad = autodiff_module()
    st, ctx = loaded_scene(mf)
    theta0 = ad.current_parameters(ctx)
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    fc = ad.mean_cutting_force(theta, ctx, 0, WINDOW)
    mean, _ = ctx.tangent_mean_force(0, WINDOW, -1)
    assert math.isclose(float(fc.detach()), mean[0], rel_tol=0, abs_tol=0)
    (2.0 * fc).backward()
    _, d6 = ctx.tangent_mean_force_all(0, WINDOW)
    for k in range(6):
        assert float(theta.grad[k]) == 2.0 * d6[k, 0], ad.PARAMS[k]


def test_all_six_directions_in_one_pass(mf):
    """Six tangent directions carried together: the value and each direction's derivatives are
    those of the single-direction pass. Each direction's arithmetic is the same expression,
    independent of the others, so they are expected bit for bit; the derivative tolerance 1e-9
    leaves room only for a different fused multiply-add contraction grown over the window."""
    st, ctx = loaded_scene(mf)
    mean6, d6 = ctx.tangent_mean_force_all(0, WINDOW)
    mean1, _ = ctx.tangent_mean_force(0, WINDOW, -1)
    np.testing.assert_allclose(mean6, mean1, rtol=1e-13, atol=0.0)
    assert d6.shape == (6, 2)
    for k in range(6):
        _, d = ctx.tangent_mean_force(0, WINDOW, k)
        np.testing.assert_allclose(d6[k], d, rtol=1e-9, atol=1e-9 * np.abs(d).max())
        assert np.abs(d6[k, 0]) > 0.0, k


def test_unsupported_settings_are_rejected(mf):
    st, ctx = loaded_scene(mf)
    ctx.set_options(mf.THERMAL_PSE, mf.JC_JOHNSON_COOK, mf.PRECISION_FP64)
    with pytest.raises(mf.MfError):
        ctx.tangent_mean_force(0, 5, 0)
    with pytest.raises(mf.MfError):
        ctx.tangent_mean_force_all(0, 5)
    ctx.set_options(mf.THERMAL_BROOKSHAW, mf.JC_TANH, mf.PRECISION_FP64)
    with pytest.raises(mf.MfError):
        ctx.tangent_mean_force(0, 5, 0)
