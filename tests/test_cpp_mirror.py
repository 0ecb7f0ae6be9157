"""The header-only C++ mirror of the reference's host API (include/mfree_cpp.hpp) compiles and
links against the library: the driver loop of the reference's mfree_gpu.cpp:146-323 written with
the mirror's names, on each of the three scenes of benchmarks.cpp, built on the CPU; and, on the
GPU, a run of that loop compared with the same steps taken through the C ABI.
"""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

DRIVER = r"""
#include <cstdio>
#include "mfree_cpp.hpp"

int main(int argc, char **) {
  grid_base *grid = nullptr;
  particle_gpu *particles;
  if (argc > 2)
    particles = setup_rings(40, &grid);
  else if (argc > 1)
    particles = setup_impact(30, &grid);
  else
    particles = setup_ref_cut(30, &grid, 10., 8., 0.002, 83.333328e-5 / 500. * 70., 0.01);
  if (global_tool == 0) global_tool = new tool();  // as the reference's main does
  leap_frog *stepper = new leap_frog(particles->N, grid->num_cell());
  int last_step = (int)(global_t_final / global_dt), freq = last_step / 135;
  for (int step = 0; step < last_step + 1; step++) {
    if (freq > 0 && step % freq == 0) {
      vtk_writer_write(particles, step / freq);
      if (global_tool) {
        vtk_writer_write(global_tool, step / freq);
        float2_t f = report_force(particles);
        std::printf("%.9g %.9g\n", f.x, f.y);
      }
    }
    stepper->step(particles, grid);
  }
  return 0;
}
"""


def test_mirror_driver_compiles_and_links(mf, tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    lib = Path(mf.LIB_PATH)
    out = tmp_path / "driver"
    cmd = [gxx, "-std=c++17", "-Wall", "-I", str(ROOT / "include"), str(src), "-L", str(lib.parent),
           "-l" + lib.stem[len("lib"):], "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert out.exists()


RUN_DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "mfree_cpp.hpp"

// the reference's driver loop (mfree_gpu.cpp:206-308) for a fixed number of steps, printing
// report_force after every step
int main(int argc, char **argv) {
  const int steps = argc > 1 ? std::atoi(argv[1]) : 10;
  grid_base *grid = nullptr;
  // the colliding rings (benchmarks.cpp:161-253): in motion from the first step
  particle_gpu *particles = setup_rings(40, &grid);
  if (global_tool == 0) global_tool = new tool();
  leap_frog *stepper = new leap_frog(particles->N, grid->num_cell());
  for (int step = 0; step < steps; step++) {
    stepper->step(particles, grid);
    float2_t f = report_force(particles);
    std::printf("F %.17g %.17g\n", f.x, f.y);
  }
  // the end state's velocities (particle_gpu holds the C ABI context)
  std::vector<double> vel(2 * (size_t)particles->N);
  if (mf_get_field(particles->ctx, MF_FIELD_VEL, vel.data()) != MF_OK) return 3;
  for (double v : vel) std::printf("V %.17g\n", v);
  return 0;
}
"""


@pytest.mark.gpu
def test_mirror_driver_runs_and_matches_the_c_abi(mf, tmp_path):
    """The mirror's driver loop, run for 200 steps of the colliding rings (setup_rings(40)),
    gives the tool force of every step (zero: no tool) and the end state's velocities of the
    same steps taken through the C ABI, bit for bit."""
    import numpy as np

    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "run_driver.cpp"
    src.write_text(RUN_DRIVER)
    lib = Path(mf.LIB_PATH)
    out = tmp_path / "run_driver"
    cmd = [gxx, "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(src), "-L", str(lib.parent),
           "-l" + lib.stem[len("lib"):], "-Wl,-rpath," + str(lib.parent), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    steps = 200
    r = subprocess.run([str(out), str(steps)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    mirror = np.array([[float(v) for v in ln.split()[1:]] for ln in lines if ln.startswith("F ")])
    mirror_vel = np.array([float(ln.split()[1]) for ln in lines if ln.startswith("V ")])
    assert mirror.shape == (steps, 2)
    sc = mf.Scene.rings(40)
    ctx = mf.Context(0)
    ctx.upload_scene(sc, mf.GRID_GREEN)
    abi = []
    for _ in range(steps):
        ctx.step(1)
        abi.append(ctx.report_force())
    vel = ctx.get("vel").reshape(-1)
    ctx.close()
    abi = np.array(abi)
    assert np.array_equal(mirror.view(np.uint64), abi.view(np.uint64))
    assert mirror_vel.shape == vel.shape
    assert np.array_equal(mirror_vel.view(np.uint64), vel.view(np.uint64))
    assert np.abs(vel).max() > 0.0  # the particles have started to move
