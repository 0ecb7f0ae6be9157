"""bench.py's reference arm runs on the host cores alone, so its one JSON line is checked here on
the CPU: the keys the benchmark contract asks of it, on the small (~6k-particle) configuration."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_one_contract_line(mf, orc):
    import scene_file

    scene_file.build_scene_files(("c1",))  # the arm's inputs (written by build() on a GPU machine)
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--config", "c1", "--steps", "2",
                        "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "dtype",
              "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["value"] > 0 and line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["cores"] >= 1
    assert cb["kind"] == ("reference" if orc.ref() is not None else "port")
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["n_particles"] == 6149


def test_reference_arm_does_not_load_the_product(mf, orc):
    """The reference arm reads its scene from the scene file: the product library is never
    loaded in its process (checked with the process's own memory map)."""
    import scene_file

    scene_file.build_scene_files(("c1",))
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--config', 'c1', '--steps', '1', "
            "'--warmup', '1']\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\nexcept SystemExit:\n    pass\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('PRODUCT_LOADED' if 'libmfree_b200' in maps else 'PRODUCT_NOT_LOADED')")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "PRODUCT_NOT_LOADED" in r.stdout, r.stdout[-2000:]


def test_benchmark_workloads_are_the_configurations(mf):
    """The scenes bench.py times: particle counts (workpiece + sampled tool particles), heat
    solver and time step of c1, c2 (the headline) and c3, as the measurements quote them."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("mfree_bench_workloads", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    expected = {"c1": (6149, 0, mf.THERMAL_BROOKSHAW, 1.1752e-3), "c2": (152796, 23899, mf.THERMAL_BROOKSHAW, 2.3505e-4),
                "c3": (499230, 78325, mf.THERMAL_PSE, 1.3012e-4)}
    for name, (n_wp, n_tool, solver, dt) in expected.items():
        p, s, _ = bench.config_params(mf, name)
        sc = mf.Scene.from_params(p)
        assert (sc.s.n_workpiece, sc.s.n_tool, s) == (n_wp, n_tool, solver), name
        assert abs(sc.s.dt - dt) < 1e-4 * dt, name
