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


def config5_context(mf):
    """Benchmark configuration 5: the cut at dx = 7.7 um (260 x 78 lattice + sampled tool
    particles, 23,416), Brookshaw, thermal contact, plain FP64 forward."""
    import bench

    p = bench.cut_params(mf, nx=260, ny=78, dx=7.7e-4)
    sc = mf.Scene.from_params(p)
    ctx = mf.Context(0)
    ctx.upload_scene(sc, mf.GRID_GREEN)
    ctx.set_options(mf.THERMAL_BROOKSHAW, mf.JC_JOHNSON_COOK, mf.PRECISION_FP64)
    return ctx


def test_config5_gradient_while_elastic(mf):
    """Configuration 5's scene over the steps before its first particle yields: the tool force
    averaged over steps 1,000-2,000 (the tool in contact, friction acting) and its derivatives
    with respect to JC A, B, n, C, m and mu in one six-direction pass. The Johnson-Cook
    derivatives are zero, as their central differences are (no particle reaches the yield
    surface); d/dmu agrees with the FP64 central difference at a relative step of 1e-4 within
    1e-3 relative. (Over the configuration's own window, steps 3,001-5,000, where the chip
    starts to yield, the central differences at relative steps 1e-3, 1e-4 and 1e-5 disagree
    with each other for A, C and mu: the objective is not differentiable at those scales.)"""
    ad = autodiff_module()
    ctx = config5_context(mf)
    theta0 = ad.current_parameters(ctx)
    skip, window = 1000, 1000
    mean, d6 = ctx.tangent_mean_force_all(skip, window)
    assert mean[0] != 0.0
    fds = []
    for k in range(6):
        h = 1e-4 * abs(theta0[k])
        th = list(theta0)
        th[k] += h
        ad.apply_parameters(ctx, th)
        fp, _ = ctx.tangent_mean_force(skip, window, -1)
        th[k] -= 2 * h
        ad.apply_parameters(ctx, th)
        fm, _ = ctx.tangent_mean_force(skip, window, -1)
        ad.apply_parameters(ctx, theta0)
        fds.append((fp - fm) / (2 * h))
    for k in range(5):  # A, B, n, C, m
        assert np.all(d6[k] == 0.0) and np.all(fds[k] == 0.0), ad.PARAMS[k]
    rel = np.abs(d6[5] - fds[5]) / np.abs(fds[5])
    assert np.all(rel <= 1e-3), (d6[5], fds[5], rel)
    ctx.close()
