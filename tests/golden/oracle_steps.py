"""Regression fixtures of the oracle's own FP64 step (test infrastructure).

The reference's step has no CPU path; its CUDA build runs on a GPU only (oracle/_ref, pinned
there and through tests/golden/ref_gpu_steps.npz). These fixtures of the oracle's own outputs
hold its whole step fixed on the benchmark configurations, on any host: c1 (143 x 43,
adiabatic, no tool particles, ~6k particles) after one step (full arrays) and after 1,000 steps (digest), and c2
(the ~150k-particle cut) after one step (digest). Every per-particle result of the oracle is
independent of the OpenMP thread count (particles are computed independently; the cell sort is
stable), so the digests hold on any host of this image. The tool force's reduction is left out
(its order follows the threads).

Written by tests/golden/make_golden.py (`python tests/golden/make_golden.py oracle`), checked by
tests/test_oracle_golden.py.
"""
from __future__ import annotations

import hashlib
import importlib.util
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
DIGEST_FIELDS = ("pos", "vel", "S", "rho", "T", "eps_pl", "eps_pl_dot", "fc", "ft", "n", "pos_t", "vel_t",
                 "S_t", "rho_t", "T_t", "blanked", "idx")
ARRAY_FIELDS = ("pos", "S", "T", "eps_pl")


def _bench():
    name = "mfree_bench_configs"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def digest(o) -> str:
    h = hashlib.sha256()
    for f in DIGEST_FIELDS:
        h.update(f.encode())
        h.update(np.ascontiguousarray(o.get(f)).tobytes())
    return h.hexdigest()


def run(mf, orc, config: str, steps: int):
    """The oracle after `steps` steps of a benchmark configuration from its initial scene."""
    bench = _bench()
    sys.path.insert(0, str(ROOT / "tests"))
    from helpers import load_oracle

    params, solver, _ = bench.config_params(mf, config)
    scene = mf.Scene.from_params(params)
    o = load_oracle(orc, bench.scene_state(mf, scene), thermal_solver=solver)
    if o.L.orc_steps(o.s, steps) != 0:
        raise RuntimeError(f"oracle steps failed on {config}")
    return o


def compute(mf, orc) -> dict:
    out = {}
    o = run(mf, orc, "c1", 1)
    for f in ARRAY_FIELDS:
        out["c1_step1_" + f] = o.get(f)
    out["c1_step1_sha256"] = np.array(digest(o))
    out["c1_step1000_sha256"] = np.array(digest(run(mf, orc, "c1", 1000)))
    out["c2_step1_sha256"] = np.array(digest(run(mf, orc, "c2", 1)))
    return out
