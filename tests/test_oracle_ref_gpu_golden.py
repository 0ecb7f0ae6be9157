"""The CPU oracle against golden vectors of the reference's own FP64 CUDA step.

tests/golden/ref_gpu_steps.npz holds the state and rates after two leap_frog::step calls of the
reference's device sources, compiled unchanged for sm_100a (its Brookshaw build and its PSE
build), on a small compressive cut scene with the tool in contact (tests/golden/ref_gpu_steps.py).
Here the oracle steps the same regenerated scene on the CPU: the cell order, hashes and blanking
must be equal, rates within 1e-12 and state within 1e-11 (max|a-b| / max|b| per field: the FMA
contraction of the two builds differs), the tool force within 1e-9 of the total contact force
(thrust::reduce sums in an unspecified order). This pins the oracle's step bodies to the
reference's own outputs without a GPU.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err
from helpers import load_oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import ref_gpu_steps as G  # noqa: E402

RATES = ("pos_t", "vel_t", "S_t", "rho_t", "T_t")
STATE = ("pos", "vel", "S", "rho", "T", "fc", "ft")


@pytest.mark.parametrize("solver", list(G.SOLVERS))
def test_oracle_equals_the_reference_gpu_step(mf, orc, solver):
    g = np.load(GOLDEN / "ref_gpu_steps.npz")
    st = G.state(mf)
    assert st["N"] == int(g[f"{solver}_N"])
    assert G.digest(st) == str(g[f"{solver}_input_digest"])  # the same input as on the GPU
    o = load_oracle(orc, st, thermal_solver=G.SOLVERS[solver])
    for _ in range(G.STEPS):
        o.L.orc_step(o.s)
    for k in G.INDEX_FIELDS:
        assert np.array_equal(o.get(k), g[f"{solver}_{k}"]), k
    nb = g[f"{solver}_blanked"] == 0.0
    for fields, tol in ((RATES, 1e-12), (STATE, 1e-11)):
        for k in fields:
            a, b = o.get(k)[nb], g[f"{solver}_{k}"][nb]
            assert np.isfinite(a).all() and np.isfinite(b).all(), k
            assert rel_err(a, b) <= tol, (k, rel_err(a, b))
    fc, ft = g[f"{solver}_fc"], g[f"{solver}_ft"]
    total = np.abs(fc).sum() + np.abs(ft).sum()
    assert np.count_nonzero(np.abs(fc).sum(axis=1)) > 5
    assert np.all(np.abs(o.report_force() - g[f"{solver}_force"]) <= 1e-9 * total)
    if solver == "pse":
        assert np.count_nonzero(g["pse_T_t"]) > 50  # heat flowed
