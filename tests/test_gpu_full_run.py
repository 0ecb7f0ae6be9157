"""Full runs of the plain FP64 step against the oracle.

The small orthogonal cut of the benchmark family (2.0 x 0.6 mm workpiece, 143 x 43 lattice,
dx = 14 um, Ti6Al4V, rake 0, clearance 7, edge radius 5 um, depth of cut 50 um, 70 m/min,
mu = 0.35, CFL 0.3) for 10,000 leap-frog steps, adiabatic without tool particles and with the
Brookshaw solver plus sampled tool particles. The tool first touches the workpiece after ~1,000
steps; by the end ~70 particles have yielded and moved above the uncut surface (the chip).

Acceptance for full runs (the single-step bar is 1e-12 per field, tested elsewhere): the
time-averaged cutting and feed force, the peak temperature rise and the chip plastic strain
(maximum and mean over the particles above the uncut surface) within 1 % of the oracle.
"""
import numpy as np
import pytest

import bench
from helpers import load_oracle, load_product, scene_state

pytestmark = pytest.mark.gpu

STEPS = 10_000


def small_cut(mf, thermal):
    p = bench.cut_params(mf, nx=143, ny=43, dx=1.4e-3)
    p.sample_tool = 1 if thermal else 0
    p.use_thermals = 1 if thermal else 0
    return scene_state(mf, mf.Scene.from_params(p))


def summary(get, st, forces):
    wp = (np.asarray(get("tool_p")) == 0.0) & (np.asarray(get("blanked")) == 0.0)
    y_top = st["pos"][st["tool_p"] == 0.0, 1].max()
    chip = wp & (np.asarray(get("pos"))[:, 1] > y_top)
    eps = np.asarray(get("eps_pl"))
    T = np.asarray(get("T"))
    return {
        "Fc": forces[:, 0].mean(), "Ff": forces[:, 1].mean(),
        "dT_peak": T[wp].max() - st["trml_wp"].T_init if st["trml_wp"].alpha != 0 else 0.0,
        "eps_chip_max": eps[chip].max() if chip.any() else 0.0,
        "eps_chip_mean": eps[chip].mean() if chip.any() else 0.0,
        "n_chip": int(chip.sum()),
    }


@pytest.mark.parametrize("thermal", [False, True])
def test_full_run_fp64_against_oracle(mf, orc, thermal):
    st = small_cut(mf, thermal)
    ctx = load_product(mf, st, thermal_solver=0)
    o = load_oracle(orc, st, thermal_solver=0)
    ctx.step(STEPS)
    f_gpu = ctx.force_log()
    f_orc = o.steps_force_log(STEPS)
    assert f_gpu.shape == (STEPS, 2)
    a = summary(ctx.get, st, f_gpu)
    b = summary(o.get, st, f_orc)
    # the run really cuts: contact, yielding and a chip
    assert b["n_chip"] > 20 and b["eps_chip_max"] > 0.05 and abs(b["Fc"]) > 0
    if thermal:
        assert b["dT_peak"] > 10.0
    for k in ("Fc", "Ff", "dT_peak", "eps_chip_max", "eps_chip_mean"):
        if b[k] == 0.0:
            assert a[k] == 0.0, k
            continue
        assert abs(a[k] - b[k]) <= 0.01 * abs(b[k]), (k, a[k], b[k])
