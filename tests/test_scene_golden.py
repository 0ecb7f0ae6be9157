"""The product's host code against the reference: setup_ref_cut, the tool, the grid box.

All of it runs on the CPU through the C ABI (no device needed for the host scene code).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import bits_equal

SCENES = ("ref_cut_default", "ref_cut_ny12_rake0", "ref_cut_sharp")
ARRAYS = ("pos", "vel", "rho", "T", "h", "fixed", "tool_p")


def scene_constants(mf, s):
    v = [getattr(s.phys, f) for f, _ in mf.Phys._fields_]
    v += [getattr(s.corr, f) for f, _ in mf.Corr._fields_]
    v += [getattr(s.joco, f) for f, _ in mf.Joco._fields_]
    v += [getattr(s.trml_wp, f) for f, _ in mf.Trml._fields_]
    v += [getattr(s.trml_tool, f) for f, _ in mf.Trml._fields_]
    v += [s.dt, s.t_final, s.tool.contact_alpha, 1.0]
    return np.array(v)


@pytest.mark.parametrize("name", SCENES)
def test_setup_ref_cut_bitwise(mf, golden, name):
    g = golden(name)
    sc = mf.Scene.ref_cut(*[float(x) if i else int(x) for i, x in enumerate(g["args"])])
    assert sc.N == int(g["N"])
    for k in ARRAYS:
        assert bits_equal(sc.array(k).reshape(-1), g[k]), k
    assert bits_equal(scene_constants(mf, sc.s), g["constants"])
    t = mf.tool_to_array(sc.s.tool)
    assert bits_equal(t["seg"], g["tool_seg"])
    assert bits_equal(t["fillet"], g["tool_fillet"])
    assert bits_equal(t["vel"], g["tool_vel"])
    assert t["mu"] == g["tool_misc"][2]
    assert sc.s.tool.slave_mass == sc.s.phys.mass


@pytest.mark.parametrize("name", SCENES)
def test_grid_box_gives_reference_geometry(mf, orc, golden, name):
    """The scene's box through grid_base::set_geometry (grid.cu:139-158) = the reference grid."""
    g = golden(name)
    sc = mf.Scene.ref_cut(*[float(x) if i else int(x) for i, x in enumerate(g["args"])])
    o = orc.Oracle(sc.N)
    s = sc.s
    o.L.orc_set_grid_locked(o.s, 0, s.grid_bbmin[0], s.grid_bbmin[1], s.grid_bbmax[0], s.grid_bbmax[1], s.grid_h)
    geo = o.geometry()
    nx, ny, bx0, by0, bx1, by1, dx, nc, locked = g["grid"]
    assert (geo["nx"], geo["ny"], geo["num_cell"]) == (int(nx), int(ny), int(nc))
    assert bits_equal([geo["bbmin_x"], geo["bbmin_y"], geo["bbmax_x"], geo["bbmax_y"], geo["dx"]],
                      [bx0, by0, bx1, by1, dx])


def test_tool_construct_sample_translate(mf, golden):
    g = golden("ref_tools")
    k = 0
    while f"t{k}_seg" in g:
        a = g[f"t{k}_args"]
        t = mf.tool_construct((a[0], a[1]), a[2], a[3], a[4], a[5], a[6], a[7])
        arr = mf.tool_to_array(t)
        assert bits_equal(arr["seg"], g[f"t{k}_seg"]), k
        assert bits_equal(arr["fillet"], g[f"t{k}_fillet"]), k
        xy = mf.tool_sample(t, 0.0014)
        assert bits_equal(xy, g[f"t{k}_sample"]), k
        t.vel[0], t.vel[1] = 1.16667e-4, 0.0
        for _ in range(50):
            mf.tool_translate(t, 1.17e-3)
        arr = mf.tool_to_array(t)
        assert bits_equal(arr["seg"], g[f"t{k}_seg_moved"]), k
        if t.has_fillet:
            assert bits_equal(arr["fillet"], g[f"t{k}_fillet_moved"]), k
        k += 1
    assert k == 4


def test_generalised_scene_explicit_lattice(mf):
    """The benchmark scenes: explicit nx x ny lattice, jitter, tool front placed at x."""
    p = mf.reference_cut_params()
    p.nx_lattice, p.ny, p.dx = 143, 43, 1.4e-3
    p.lo_x, p.lo_y = 0.0, 0.0
    p.jitter, p.seed = 0.005, 1
    p.tool_front_x = -0.1 * 1.4e-3
    p.feed, p.rake, p.clear, p.chamfer = 0.005, 0.0, 7.0, 5e-4
    p.cfl = 0.3
    p.sample_tool = 0
    p.use_thermals = 0
    sc = mf.Scene.from_params(p)
    assert sc.s.n_workpiece == 143 * 43 and sc.s.n_tool == 0
    pos = sc.array("pos")
    lattice_x = np.repeat(np.arange(143) * 1.4e-3, 43)
    assert np.max(np.abs(pos[:, 0] - lattice_x)) <= 0.005 * 1.4e-3 * (1 + 1e-12)
    # deterministic
    sc2 = mf.Scene.from_params(p)
    assert bits_equal(sc2.array("pos"), pos)
    # bottom row fixed
    fixed = sc.array("fixed")
    assert np.all(fixed.reshape(143, 43)[:, 0] == 1.0)
    # tool front at the requested x, low point at hi_y - feed
    t = mf.tool_to_array(sc.s.tool)
    hi_y = 42 * 1.4e-3
    low = t["fillet"][4] - t["fillet"][0]
    assert abs(low - (hi_y - 0.005)) < 1e-12
    # dt = cfl*hdx*dx/(sqrt(K/rho0) + sqrt(v))
    s = sc.s
    assert abs(s.dt - 0.3 * 1.5 * 1.4e-3 / (np.sqrt(s.phys.K / s.phys.rho0) + np.sqrt(s.speed))) < 1e-18


# (tl_x, tl_y, length, height, rake, clear, r, mu), as tests/golden/make_golden.py's TOOLS
VTK_TOOLS = [
    (-0.046, 0.0986074, 0.0413176, 0.0431, 10.0, 8.0, 0.002, 0.35),
    (-0.046, 0.0986074, 0.0413176, 0.0431, 0.0, 7.0, 0.0005, 0.35),
    (-0.046, 0.0986074, 0.0413176, 0.0431, -10.0, 6.0, 0.001, 0.2),
    (0.0, 0.01, 0.02, 0.02, 15.0, 8.0, 0.0, 0.35),
]


@pytest.mark.parametrize("k", range(len(VTK_TOOLS)))
def test_tool_vtk_file_byte_equal(mf, golden, tmp_path, k):
    """mf_vtk_write_tool against the reference's own vtk_writer_write(const tool*, int)
    (vtk_writer.cpp:185-264), as built and after a translation."""
    g = golden("ref_vtk_tool")
    t = VTK_TOOLS[k]
    tool = mf.tool_construct((t[0], t[1]), *t[2:])
    mf.vtk_write_tool(tool, tmp_path / "built.vtk")
    assert (tmp_path / "built.vtk").read_bytes() == bytes(g[f"t{k}_built"])
    tool.vel[0], tool.vel[1] = -1.16667e-4, 0.0
    mf.tool_translate(tool, 37.5)
    mf.vtk_write_tool(tool, tmp_path / "moved.vtk")
    assert (tmp_path / "moved.vtk").read_bytes() == bytes(g[f"t{k}_moved"])


def test_particle_vtk_file_byte_equal(mf, golden, tmp_path):
    """The particle VTK writer (shared by mf_vtk_write_particles and its asynchronous form)
    against the reference's own vtk_writer_write(const particle_gpu*, int)
    (vtk_writer.cpp:20-178) on the same host arrays, every particle unblanked."""
    g = golden("ref_vtk_particles")
    fields = {k: g[k] for k in ("pos", "vel", "rho", "p", "T", "eps_pl", "S", "fixed", "tool_p")}
    fields["blanked"] = np.zeros(len(g["rho"]))
    mf.vtk_write_particle_arrays(tmp_path / "p.vtk", fields)
    assert (tmp_path / "p.vtk").read_bytes() == bytes(g["vtk"])


VALIDATION = ("ref_rings_nbox40", "ref_rings_nbox21", "ref_impact_nbox30", "ref_impact_nbox17")


@pytest.mark.parametrize("name", VALIDATION)
def test_validation_scenes_bitwise(mf, orc, golden, name):
    """mf_scene_setup_rings / mf_scene_setup_impact against the reference's own setup_rings /
    setup_impact (benchmarks.cpp:161-253, 23-159): arrays, constants, time step and grid."""
    g = golden(name)
    kind, nbox = str(g["kind"]), int(g["nbox"])
    sc = (mf.Scene.rings if kind == "rings" else mf.Scene.impact)(nbox)
    s = sc.s
    assert sc.N == int(g["N"]) and s.n_workpiece == sc.N and s.n_tool == 0
    for k in ARRAYS:
        assert bits_equal(sc.array(k).reshape(-1), g[k]), k
    c = scene_constants(mf, s)
    c[-1] = float(s.has_joco)  # rings set no Johnson-Cook constants (no plasticity)
    assert bits_equal(c, g["constants"])
    assert s.has_joco == (1 if kind == "impact" else 0)
    assert s.tool.num_seg == 0 and s.tool.has_fillet == 0
    locked = bool(g["grid"][8])
    assert s.grid_max_cell == int(g["grid_max_cell"])
    assert locked == (s.grid_max_cell == 0) == (kind == "rings")
    if locked:  # the box through grid_base::set_geometry gives the reference's grid
        o = orc.Oracle(sc.N)
        o.L.orc_set_grid_locked(o.s, 0, s.grid_bbmin[0], s.grid_bbmin[1], s.grid_bbmax[0], s.grid_bbmax[1],
                                s.grid_h)
        geo = o.geometry()
        nx, ny, bx0, by0, bx1, by1, dx, nc, _ = g["grid"]
        assert (geo["nx"], geo["ny"], geo["num_cell"]) == (int(nx), int(ny), int(nc))
        assert bits_equal([geo["bbmin_x"], geo["bbmin_y"], geo["bbmax_x"], geo["bbmax_y"], geo["dx"]],
                          [bx0, by0, bx1, by1, dx])
    else:
        assert s.grid_max_cell == 10 * sc.N


@pytest.mark.parametrize("nbox", [-3, 0, 1])
def test_validation_scenes_refuse_degenerate_lattices(mf, nbox):
    for make in (mf.Scene.rings, mf.Scene.impact):
        with pytest.raises(mf.MfError) as e:
            make(nbox)
        assert e.value.code == -1  # MF_ERR_INVALID


@pytest.mark.parametrize("kind", ["rings", "impact"])
def test_validation_scenes_live_against_the_reference(mf, orc, kind):
    """The same comparison live, against the reference's own setup compiled on this host, over a
    range of lattice sizes (odd and even nbox, coarse to fine)."""
    R = orc.ref()
    if R is None:
        pytest.skip("the reference's sources were not built here")
    setup = R.refh_setup_rings if kind == "rings" else R.refh_setup_impact
    make = mf.Scene.rings if kind == "rings" else mf.Scene.impact
    for nbox in (5, 8, 13, 24, 37, 50, 64):
        n = setup(nbox)
        if n == 0:  # (nbox 5: no lattice point in the rings) an empty scene is refused
            with pytest.raises(mf.MfError):
                make(nbox)
            continue
        sc = make(nbox)
        assert sc.N == n, nbox
        for k, f in enumerate(ARRAYS):
            ref = np.zeros(n * (2 if f in ("pos", "vel") else 1))
            R.refh_get_array(k, ref.ctypes.data_as(C.c_void_p))
            assert bits_equal(sc.array(f).reshape(-1), ref), (nbox, f)
        c = np.zeros(64)
        m = R.refh_get_constants(c.ctypes.data_as(C.c_void_p))
        mine = scene_constants(mf, sc.s)
        mine[-1] = float(sc.s.has_joco)
        assert bits_equal(mine, c[:m]), nbox
        assert sc.s.grid_max_cell == R.refh_get_grid_max_cell(), nbox
