"""Shared fixtures: the product package (through its C ABI), the oracle and the golden data.

Tests marked ``gpu`` need a CUDA device and the sm_100a library; everything else runs on
the CPU. The oracle (oracle/) is used here only as the checker.
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "mfree_iwf-ul_cut_gpu_b200"
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the sm_100a library")


def load_product():
    name = "mfree_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def mf():
    sys.path.insert(0, str(PKG_DIR))
    import build as pkg_build  # mfree_iwf-ul_cut_gpu_b200/build.py
    pkg_build.build()
    return load_product()


@pytest.fixture(scope="session")
def orc():
    import binding
    import build_oracle
    build_oracle.build_oracle()
    return binding


@pytest.fixture(scope="session")
def c2_midcut(mf, tmp_path_factory):
    """GPU: the ~150k-particle benchmark cut (176,695 particles, Brookshaw) after 0.05 mm of
    plain FP64 cut (~182k steps), saved once per session to a state file; returns the scene,
    its thermal solver, the file and the number of steps taken."""
    import bench

    p, solver, _ = bench.config_params(mf, "c2")
    sc = mf.Scene.from_params(p)
    ctx = mf.Context(0)
    ctx.upload_scene(sc, mf.GRID_GREEN)
    ctx.set_options(solver, mf.JC_JOHNSON_COOK, mf.PRECISION_FP64)
    s = sc.s
    steps = int(round(0.005 / (s.tool.vel[0] * s.dt)))
    ctx.step(steps)
    ctx.synchronize()
    path = tmp_path_factory.mktemp("midcut") / "c2_midcut.mfstate"
    ctx.state_save(str(path))
    st = ctx.status()
    ctx.close()
    return {"scene": sc, "solver": solver, "path": path, "steps": steps, "status": st}


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / f"{name}.npz"))
    return load


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    b = np.ascontiguousarray(np.asarray(b, dtype=np.float64))
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def rel_err(a, b) -> float:
    """Norm-wise relative error max|a-b| / max|b| (0 when both are zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b)) if b.size else 0.0
    num = np.max(np.abs(a - b)) if a.size else 0.0
    if den == 0.0:
        return float(num)
    return float(num / den)
