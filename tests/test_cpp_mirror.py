"""The header-only C++ mirror of the reference's host API (include/mfree_cpp.hpp) compiles and
links against the library: the driver loop of the reference's mfree_gpu.cpp:146-323 written with
the mirror's names, on each of the three scenes of benchmarks.cpp (CPU only: built, not run).
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
