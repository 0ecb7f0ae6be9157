"""Generate the golden fixtures in tests/golden/ from the reference's own sources.

The reference has no tests and no golden vectors of its own. These fixtures are outputs of
the reference's host-compilable sources (benchmarks.cpp setup_ref_cut, tool.cpp,
geometric_primitives.cpp, kernels.cuh, plasticity.cuh), compiled where they lie by
oracle/build_oracle.py into oracle/_ref/libref_host.so, on seeded inputs. They pin the
oracle and the product's host code on machines where the reference tree is absent.

    python tests/golden/make_golden.py              # every fixture
    python tests/golden/make_golden.py validation   # the rings and impact scenes only
    python tests/golden/make_golden.py oracle       # the oracle's own step (oracle_steps.npz)
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))

import binding as B  # noqa: E402
import build_oracle  # noqa: E402

SPEED_70 = 83.333328e-5 / 500.0 * 70.0
SCENES = {
    # name: setup_ref_cut(ny, rake, clear, chamfer, speed, feed)
    "ref_cut_default": (30, 10.0, 8.0, 0.002, SPEED_70, 0.01),
    "ref_cut_ny12_rake0": (12, 0.0, 7.0, 0.0005, 1.16667e-4, 0.005),
    "ref_cut_sharp": (16, 5.0, 8.0, 0.0, SPEED_70, 0.01),
}
VALIDATION = {
    # name: (setup function, nbox)
    "ref_rings_nbox40": ("rings", 40),
    "ref_rings_nbox21": ("rings", 21),
    "ref_impact_nbox30": ("impact", 30),
    "ref_impact_nbox17": ("impact", 17),
}
JC_REF = [0.00862, 0.00331, 0.01, 0.34, 0.8, 1836.0, 300.0, 1e-6, 1.1, 0.4, 12.0, 1.0]
TOOLS = [
    # tl_x, tl_y, length, height, rake, clear, r, mu
    (-0.046, 0.0986074, 0.0413176, 0.0431, 10.0, 8.0, 0.002, 0.35),
    (-0.046, 0.0986074, 0.0413176, 0.0431, 0.0, 7.0, 0.0005, 0.35),
    (-0.046, 0.0986074, 0.0413176, 0.0431, -10.0, 6.0, 0.001, 0.2),
    (0.0, 0.01, 0.02, 0.02, 15.0, 8.0, 0.0, 0.35),
]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def scene(R, name, args):
    n = R.refh_setup_ref_cut(*args)
    out = {"args": np.array(args, dtype=np.float64), "N": np.array(n)}
    for k, f in enumerate(["pos", "vel", "rho", "T", "h", "fixed", "tool_p"]):
        w = 2 if f in ("pos", "vel") else 1
        a = np.zeros(n * w)
        R.refh_get_array(k, _p(a))
        out[f] = a
    c = np.zeros(64)
    k = R.refh_get_constants(_p(c))
    out["constants"] = c[:k]
    g = np.zeros(9)
    R.refh_get_grid(_p(g))
    out["grid"] = g
    seg, fil, misc, vel = np.zeros(55), np.zeros(5), np.zeros(3), np.zeros(2)
    ns = R.refh_get_scene_tool(_p(seg), _p(fil), _p(misc), _p(vel))
    out["tool_seg"] = seg.reshape(5, 11)[:ns]
    out["tool_fillet"] = fil
    out["tool_misc"] = misc
    out["tool_vel"] = vel
    np.savez_compressed(HERE / f"{name}.npz", **out)
    return n


def kernels(R, rng):
    m = 4000
    h = rng.uniform(1e-4, 1e-2, m)
    xi = rng.uniform(-0.1, 0.1, m)
    yi = rng.uniform(-0.1, 0.1, m)
    r = h * rng.uniform(0.0, 2.2, m)
    a = rng.uniform(0, 2 * np.pi, m)
    xj, yj = xi + r * np.cos(a), yi + r * np.sin(a)
    # exact boundary cases: r^2 == 4h^2 side, tiny separations
    xj[:20] = xi[:20] + 2 * h[:20]
    yj[:20] = yi[:20]
    xj[20:40] = xi[20:40] + 1e-5
    yj[20:40] = yi[20:40]
    w = np.zeros((m, 3))
    pse = np.zeros(m)
    o = np.zeros(3)
    for i in range(m):
        R.refh_cubic_spline(xi[i], yi[i], xj[i], yj[i], h[i], _p(o))
        w[i] = o
        pse[i] = R.refh_lapl_pse(xi[i], yi[i], xj[i], yj[i], h[i])
    np.savez_compressed(HERE / "ref_kernels.npz", xi=xi, yi=yi, xj=xj, yj=yj, h=h, w=w, pse=pse)


def plasticity(R, rng):
    jc = np.array(JC_REF)
    m = 1500
    eps = rng.uniform(0, 2.0, m)
    eps[:10] = 0.0
    epsdot = 10 ** rng.uniform(-9, -3, m)
    epsdot[10:20] = 0.0
    T = rng.uniform(300, 1500, m)
    T[20:25] = 300.0
    sy = np.array([R.refh_sigma_yield(_p(jc), eps[i], epsdot[i], T[i]) for i in range(m)])
    syt = np.array([R.refh_sigma_yield_tanh(_p(jc), eps[i], epsdot[i], T[i]) for i in range(m)])
    norm = rng.uniform(0.005, 0.04, m)
    dt = rng.uniform(1e-4, 2e-3, m)
    init = np.maximum(epsdot * dt * np.sqrt(2.0 / 3.0), 1e-8)
    mu = 0.4074074074074074
    sec0 = np.array([R.refh_solve_secant(_p(jc), 0, init[i], 1e-6, norm[i], eps[i], T[i], dt[i], mu) for i in range(m)])
    sec1 = np.array([R.refh_solve_secant(_p(jc), 1, init[i], 1e-6, norm[i], eps[i], T[i], dt[i], mu) for i in range(m)])
    np.savez_compressed(HERE / "ref_plasticity.npz", jc=jc, eps=eps, epsdot=epsdot, T=T, sigma_yield=sy,
                        sigma_yield_tanh=syt, norm=norm, dt=dt, init=init, mu=np.array(mu), secant_jc=sec0,
                        secant_tanh=sec1)


def tools(R):
    out = {}
    for k, t in enumerate(TOOLS):
        ns = R.refh_tool_create(*t)
        seg, fil, misc = np.zeros(55), np.zeros(5), np.zeros(3)
        R.refh_tool_dump(_p(seg), _p(fil), _p(misc))
        out[f"t{k}_args"] = np.array(t)
        out[f"t{k}_seg"] = seg.reshape(5, 11)[:ns]
        out[f"t{k}_fillet"] = fil.copy()
        out[f"t{k}_misc"] = misc.copy()
        dx = 0.0014
        cap = 200000
        xy = np.zeros(2 * cap)
        n = R.refh_tool_sample(dx, _p(xy), cap)
        out[f"t{k}_sample"] = xy[: 2 * n].reshape(n, 2)
        bb = np.zeros(4)
        R.refh_tool_safe_bb(1e-3, _p(bb))
        out[f"t{k}_safe_bb"] = bb
        # 50 translations with the cutting velocity
        R.refh_tool_set_vel(1.16667e-4, 0.0)
        for _ in range(50):
            R.refh_tool_update(1.17e-3)
        seg2 = np.zeros(55)
        R.refh_tool_dump(_p(seg2), _p(fil), _p(misc))
        out[f"t{k}_seg_moved"] = seg2.reshape(5, 11)[:ns]
        out[f"t{k}_fillet_moved"] = fil.copy()
    np.savez_compressed(HERE / "ref_tools.npz", **out)


def usui_inputs(rng, n=600):
    """Seeded particle arrays for the Usui wear evaluation: about half in contact."""
    contact = rng.random(n) < 0.5
    fc = np.where(contact[:, None], rng.normal(0, 1e-4, (n, 2)), 0.0)
    ft = np.where(contact[:, None], rng.normal(0, 3e-5, (n, 2)), 0.0)
    fc[::7, 0] = 0.0  # contact seen through one component only
    ang = rng.uniform(0, 2 * np.pi, n)
    return {"pos": rng.uniform(0, 0.2, (n, 2)), "vel": rng.normal(0, 1e-4, (n, 2)), "fc": fc, "ft": ft,
            "h": rng.uniform(1e-4, 1e-3, n), "n": np.stack([np.cos(ang), np.sin(ang)], axis=1),
            "T": rng.uniform(300.0, 900.0, n), "K": np.array(1e-8), "alpha": np.array(-2500.0),
            "tool_vel": np.array([-1.16667e-4, 0.0]), "dt": np.array(0.01)}


def usui(R, rng):
    d = usui_inputs(rng)
    out = np.zeros(4)
    R.refh_usui(len(d["h"]), *[_p(np.ascontiguousarray(d[k])) for k in ("pos", "vel", "fc", "ft", "h", "n", "T")],
                C.c_double(float(d["K"])), C.c_double(float(d["alpha"])), C.c_double(d["tool_vel"][0]),
                C.c_double(d["tool_vel"][1]), C.c_double(float(d["dt"])), _p(out))
    np.savez_compressed(HERE / "ref_usui.npz", usui=out, **d)


def vtk_tools(R):
    """The reference's tool VTK file (vtk_writer.cpp:185-264) for each tool of TOOLS, as built
    and after a translation (the writer writes results/vtk_tool_<step>.vtk under the working
    directory, so it runs in a scratch directory)."""
    import os
    import tempfile

    R.refh_tool_create.argtypes = [C.c_double] * 8
    R.refh_tool_set_vel.argtypes = [C.c_double, C.c_double]
    R.refh_tool_update.argtypes = [C.c_double]
    out = {}
    cwd = os.getcwd()
    scratch = ROOT / "_work"
    scratch.mkdir(exist_ok=True)
    with tempfile.TemporaryDirectory(dir=scratch) as d:
        os.chdir(d)
        try:
            os.mkdir("results")
            for k, t in enumerate(TOOLS):
                R.refh_tool_create(*t)
                R.refh_vtk_tool(2 * k)
                R.refh_tool_set_vel(-1.16667e-4, 0.0)
                R.refh_tool_update(37.5)
                R.refh_vtk_tool(2 * k + 1)
                for step in (2 * k, 2 * k + 1):
                    data = open(f"results/vtk_tool_{step:06d}.vtk", "rb").read()
                    out[f"t{k}_{'moved' if step % 2 else 'built'}"] = np.frombuffer(data, dtype=np.uint8)
        finally:
            os.chdir(cwd)
    np.savez_compressed(HERE / "ref_vtk_tool.npz", **out)


def vtk_particles(R, rng, n=400):
    """The reference's particle VTK file (vtk_writer.cpp:20-178) for a seeded state. The
    reference never fills its blanked array (Q12); the fixture is kept only if it wrote every
    particle, so that it is the writer's output for an all-unblanked state."""
    import os
    import tempfile

    d = {"pos": rng.uniform(-0.05, 0.2, (n, 2)), "vel": rng.normal(0, 1e-4, (n, 2)),
         "rho": rng.uniform(4.3, 4.5, n), "h": np.full(n, 4.2e-4), "p": rng.normal(0, 1e-3, n),
         "T": rng.uniform(300, 900, n), "eps_pl": rng.uniform(0, 2, n), "S": rng.normal(0, 1e-2, (n, 4)),
         "fixed": (rng.random(n) < 0.1).astype(float), "tool_p": (rng.random(n) < 0.2).astype(float)}
    R.refh_vtk_particles.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 10
    cwd = os.getcwd()
    scratch = ROOT / "_work"
    scratch.mkdir(exist_ok=True)
    with tempfile.TemporaryDirectory(dir=scratch) as tdir:
        os.chdir(tdir)
        try:
            os.mkdir("results")
            R.refh_vtk_particles(3, n, *[_p(np.ascontiguousarray(d[k])) for k in
                                         ("pos", "vel", "rho", "h", "p", "T", "eps_pl", "S", "fixed", "tool_p")])
            data = open("results/vtk_out_000003.vtk", "rb").read()
        finally:
            os.chdir(cwd)
    assert f"POINTS {n} float".encode() in data, "the reference skipped particles (uninitialised blanked array)"
    np.savez_compressed(HERE / "ref_vtk_particles.npz", vtk=np.frombuffer(data, dtype=np.uint8), **d)


def validation_scene(R, name, kind, nbox):
    """setup_rings / setup_impact (benchmarks.cpp:161-253, 23-159): arrays, constants, grid."""
    n = (R.refh_setup_rings if kind == "rings" else R.refh_setup_impact)(nbox)
    out = {"kind": np.array(kind), "nbox": np.array(nbox), "N": np.array(n)}
    for k, f in enumerate(["pos", "vel", "rho", "T", "h", "fixed", "tool_p"]):
        w = 2 if f in ("pos", "vel") else 1
        a = np.zeros(n * w)
        R.refh_get_array(k, _p(a))
        out[f] = a
    c = np.zeros(64)
    k = R.refh_get_constants(_p(c))
    out["constants"] = c[:k]
    g = np.zeros(9)
    R.refh_get_grid(_p(g))
    out["grid"] = g
    out["grid_max_cell"] = np.array(R.refh_get_grid_max_cell())
    np.savez_compressed(HERE / f"{name}.npz", **out)
    return n


def oracle_fixture():
    """The oracle's own step on the benchmark configurations (tests/golden/oracle_steps.py);
    needs the product's host scene code and the oracle, not the reference."""
    import importlib.util

    import oracle_steps

    build_oracle.build_oracle()
    spec = importlib.util.spec_from_file_location("mfree_b200", ROOT / "mfree_iwf-ul_cut_gpu_b200" / "__init__.py",
                                                  submodule_search_locations=[str(ROOT / "mfree_iwf-ul_cut_gpu_b200")])
    mf = importlib.util.module_from_spec(spec)
    sys.modules["mfree_b200"] = mf
    spec.loader.exec_module(mf)
    np.savez_compressed(HERE / "oracle_steps.npz", **oracle_steps.compute(mf, B))


def ref_gpu_fixture():
    """The reference's own CUDA step on a small scene (tests/golden/ref_gpu_steps.py); needs a CUDA
    device and oracle/_ref/libref_gpu.so and libref_gpu_pse.so."""
    import importlib.util

    sys.path.insert(0, str(ROOT / "tests"))
    import ref_gpu_steps

    spec = importlib.util.spec_from_file_location("mfree_b200", ROOT / "mfree_iwf-ul_cut_gpu_b200" / "__init__.py",
                                                  submodule_search_locations=[str(ROOT / "mfree_iwf-ul_cut_gpu_b200")])
    mf = importlib.util.module_from_spec(spec)
    sys.modules["mfree_b200"] = mf
    spec.loader.exec_module(mf)
    if B.ref_gpu() is None or B.ref_gpu("pse") is None:
        raise SystemExit("the reference's GPU builds are missing (oracle/build_oracle.py on a machine with its tree)")
    np.savez_compressed(HERE / "ref_gpu_steps.npz", **ref_gpu_steps.compute(mf, B))


def main():
    if sys.argv[1:] == ["oracle"]:
        oracle_fixture()
        return
    if sys.argv[1:] == ["ref_gpu"]:
        ref_gpu_fixture()
        return
    build_oracle.build_ref()
    R = B.ref()
    if R is None:
        raise SystemExit("the reference tree is not available; fixtures cannot be regenerated here")
    for name, (kind, nbox) in VALIDATION.items():
        print(name, validation_scene(R, name, kind, nbox))
    if sys.argv[1:] == ["validation"]:
        return
    rng = np.random.default_rng(20261203)
    for name, args in SCENES.items():
        print(name, scene(R, name, args))
    kernels(R, rng)
    plasticity(R, rng)
    tools(R)
    usui(R, np.random.default_rng(77))
    vtk_tools(R)
    vtk_particles(R, np.random.default_rng(91))


if __name__ == "__main__":
    main()
