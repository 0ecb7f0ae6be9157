"""Write the benchmark configurations' initial scenes to files the baselines read.

ORACLE - test infrastructure: the scene is the workload's input (particle arrays, constants,
tool, grid and time step of the ~6k, ~150k and ~500k-particle cuts), generated once by the
project's scene setup (a generalisation of the reference's setup_ref_cut) and saved as
oracle/_build/scenes/<config>.npz, so that bench.py's reference arm (the CPU path on the host
cores) loads the same inputs without loading the product library.

    python oracle/scene_file.py [c1 c2 c3]
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SCENES = HERE / "_build" / "scenes"


def _doubles(struct):
    return np.array([getattr(struct, f) for f, _ in struct._fields_], dtype=np.float64)


def scene_path(config: str) -> Path:
    return SCENES / f"{config}.npz"


def write_scene(config: str) -> Path:
    sys.path.insert(0, str(ROOT))
    import bench

    mf = bench.load_package()
    params, solver, workload = bench.config_params(mf, config)
    sc = mf.Scene.from_params(params)
    s = sc.s
    d = {k: sc.array(k).copy() for k in ("pos", "vel", "rho", "T", "h", "fixed", "tool_p")}
    d.update(phys=_doubles(s.phys), corr=_doubles(s.corr), joco=_doubles(s.joco), trml_wp=_doubles(s.trml_wp),
             trml_tool=_doubles(s.trml_tool), dt=np.array([s.dt]),
             grid=np.array([s.grid_bbmin[0], s.grid_bbmin[1], s.grid_bbmax[0], s.grid_bbmax[1], s.grid_h]),
             tool=np.frombuffer(C.string_at(C.byref(s.tool), C.sizeof(s.tool)), dtype=np.uint8).copy(),
             thermal_solver=np.array([solver]), n_tool=np.array([s.n_tool]), n_workpiece=np.array([s.n_workpiece]))
    SCENES.mkdir(parents=True, exist_ok=True)
    out = scene_path(config)
    tmp = out.with_suffix(".tmp.npz")
    np.savez_compressed(tmp, **d)
    tmp.replace(out)
    return out


def build_scene_files(configs=("c1", "c2")) -> None:
    """The scene files of `configs` that are missing or older than the scene code."""
    src = [ROOT / "bench.py", ROOT / "mfree_iwf-ul_cut_gpu_b200" / "lib" / "libmfree_b200.so"]
    for c in configs:
        p = scene_path(c)
        if not p.exists() or any(s.exists() and s.stat().st_mtime > p.stat().st_mtime for s in src):
            write_scene(c)


if __name__ == "__main__":
    for c in (sys.argv[1:] or ["c1", "c2"]):
        print(write_scene(c))
