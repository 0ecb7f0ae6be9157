"""bench.py's comparison of saved cut runs (cut_compare) is host logic: checked here on the CPU
with synthetic runs of the small (~6k-particle) configuration — a run whose tool force turns
non-finite, forces compared over the steps both runs' forces are finite, end fields compared
only where both runs reached the planned end, the perturbed-form pairing and the block means."""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def fake_run(path, scene, forces, planned, eps_scale=1.0, blanked=0):
    N = scene.N
    rng = np.random.default_rng(len(forces))
    st = {"S": rng.normal(size=(N, 4)), "p": rng.normal(size=N), "eps_pl": eps_scale * np.ones(N),
          "T": scene.s.trml_wp.T_init + eps_scale * np.ones(N), "tool_p": scene.array("tool_p").copy(),
          "blanked": np.zeros(N), "pos": scene.array("pos").copy() + 1e-3}
    status = {"blanked": blanked, "secant_cap_hits": 0, "sorts": 7, "timeline": [[len(forces), blanked, 0]]}
    np.savez(path, forces=forces, secs=np.array([np.nan]), status=np.array([json.dumps(status)]),
             steps_planned=np.array([planned]), **{"state_" + k: v for k, v in st.items()})


def test_finite_prefix():
    f = np.ones((10, 2))
    assert bench.finite_prefix(f) == 10
    f[6, 1] = np.nan
    assert bench.finite_prefix(f) == 6
    f[0, 0] = np.inf
    assert bench.finite_prefix(f) == 0


def test_cut_compare(mf, tmp_path):
    p, _, _ = bench.config_params(mf, "c1")
    scene = mf.Scene.from_params(p)
    planned = 1000
    ref = np.tile([2.0, -1.0], (planned, 1))
    ref[600:] = np.nan  # the reference run stops being finite at step 600
    fake_run(tmp_path / "cut_fp64.npz", scene, ref[:620], planned, blanked=3)
    mixed = np.tile([2.02, -1.0], (planned, 1))
    fake_run(tmp_path / "cut_mixed.npz", scene, mixed, planned, eps_scale=1.1)
    fake_run(tmp_path / "cut_mixed_sorted.npz", scene, np.tile([2.0, -1.01], (planned, 1)), planned)
    fake_run(tmp_path / "cut_mixed@p.npz", scene, np.tile([2.04, -1.0], (planned, 1)), planned)
    out = bench.cut_compare(mf, scene, [str(tmp_path / f"cut_{n}.npz")
                                        for n in ("fp64", "mixed", "mixed_sorted", "mixed@p")])["forms"]
    f64 = out["fp64"]
    assert f64["completed"] is False and f64["first_nonfinite_force_step"] == 600 and f64["blanked"] == 3
    assert f64["block_mean_force"][5] == [2.0, -1.0] and f64["block_mean_force"][6] is None
    e = out["mixed"]["errors_against_fp64"]
    assert e["force_steps"] == 600
    assert abs(e["mean_fc_rel_err"] - 0.01) < 1e-12 and e["mean_ff_rel_err"] == 0.0
    assert e["von_mises_rel_l2"] is None and e["chip"] is None  # the FP64 run did not reach the end
    e = out["mixed"]["errors_against_mixed_sorted"]
    assert e["force_steps"] == planned and abs(e["mean_ff_rel_err"] - 0.01 / 1.01) < 1e-12
    assert abs(e["dT_peak_rel_err"] - 0.1) < 1e-12  # both runs complete: end fields compared
    assert "errors_against_unperturbed" in out["mixed@p"]
    assert abs(out["mixed@p"]["errors_against_unperturbed"]["mean_fc_rel_err"] - 0.02 / 2.02) < 1e-12
    assert "errors_against_mixed_sorted" not in out["mixed_sorted"]


def test_form_flags(mf):
    assert bench.form_flags(mf, "fp64") == (mf.PRECISION_FP64, 0)
    assert bench.form_flags(mf, "mixed") == (mf.PRECISION_MIXED, mf.OPT_NEIGHBOUR_LISTS)
    assert bench.form_flags(mf, "mixed@p") == bench.form_flags(mf, "mixed")
    assert bench.form_flags(mf, "mixed_sorted") == (mf.PRECISION_MIXED, mf.OPT_SORT_EVERY_STEP)
