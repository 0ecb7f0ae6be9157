"""Build one particle state and load it into both the product (C ABI) and the oracle.

States are derived from the reference cut scene (setup_ref_cut) and perturbed with seeded
random velocities, stresses, densities, temperatures, forces and plastic strains, with
the tool pushed into the workpiece so that contact, friction and friction heat are active.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

SCALAR = ("rho", "T", "h", "fixed", "tool_p", "eps_pl", "eps_pl_dot", "rho_t", "T_t", "blanked")
VEC2 = ("pos", "vel", "fc", "ft", "n", "pos_t", "vel_t")
VEC4 = ("S", "S_t")


def perturbed_scene(mf, ny=12, seed=0, tensile=False, blank_frac=0.0, tool_push_dx=3.0, thermal=True,
                    rake=0.0, clear=7.0, chamfer=0.0005, feed=0.005, speed=1.16667e-4):
    """A state dict from setup_ref_cut(ny, ...) with seeded perturbations."""
    sc = mf.Scene.ref_cut(ny, rake, clear, chamfer, speed, feed)
    s = sc.s
    N = sc.N
    rng = np.random.default_rng(seed)
    dx = s.grid_h / 1.5
    st = {"N": N}
    st["pos"] = sc.array("pos").copy()
    st["rho"] = sc.array("rho").copy()
    st["T"] = sc.array("T").copy()
    st["h"] = sc.array("h").copy()
    st["fixed"] = sc.array("fixed").copy()
    st["tool_p"] = sc.array("tool_p").copy()
    wp = st["tool_p"] == 0.0
    nw = int(wp.sum())
    st["pos"][wp] += rng.uniform(-0.05, 0.05, (nw, 2)) * dx
    st["vel"] = np.zeros((N, 2))
    st["vel"][wp] = rng.normal(0.0, 1e-4, (nw, 2))
    # density slightly above rho0 (compressed) keeps the principal stresses negative
    st["rho"][wp] *= 1.0 + rng.uniform(0.0005, 0.003, nw)
    st["T"] += rng.uniform(0.0, 200.0, N)
    st["S"] = np.zeros((N, 4))
    amp = 4e-3 if tensile else 1e-4
    st["S"][wp] = rng.normal(0.0, amp, (nw, 4))
    st["eps_pl"] = np.where(wp, rng.uniform(0.0, 0.5, N), 0.0)
    st["eps_pl_dot"] = np.where(wp, 10 ** rng.uniform(-8, -4, N), 0.0)
    st["fc"] = np.zeros((N, 2))
    st["ft"] = np.zeros((N, 2))
    st["ft"][wp] = rng.normal(0.0, 1e-9, (nw, 2))
    st["n"] = rng.normal(0.0, 1.0, (N, 2))
    st["n"] /= np.linalg.norm(st["n"], axis=1, keepdims=True)
    st["pos_t"] = np.zeros((N, 2))
    st["vel_t"] = np.zeros((N, 2))
    st["pos_t"][wp] = rng.normal(0.0, 1e-4, (nw, 2))
    st["vel_t"][wp] = rng.normal(0.0, 1e-3, (nw, 2))
    st["rho_t"] = np.where(wp, rng.normal(0.0, 1e-3, N), 0.0)
    st["S_t"] = np.zeros((N, 4))
    st["S_t"][wp] = rng.normal(0.0, 1e-3, (nw, 4))
    st["T_t"] = rng.normal(0.0, 1.0, N)
    st["blanked"] = np.zeros(N)
    if blank_frac > 0:
        st["blanked"][rng.random(N) < blank_frac] = 1.0
    # constants
    st["phys"], st["corr"] = s.phys, s.corr
    st["joco"] = s.joco
    st["trml_wp"] = s.trml_wp if thermal else mf.Trml()
    st["trml_tool"] = s.trml_tool if thermal else mf.Trml()
    st["dt"] = s.dt
    st["grid"] = (tuple(s.grid_bbmin), tuple(s.grid_bbmax), s.grid_h)
    tool = mf.ToolState()
    C.memmove(C.byref(tool), C.byref(s.tool), C.sizeof(mf.ToolState))
    # push the tool into the workpiece so that particles are inside it: close the gap
    # between the tool's front and the workpiece's left edge, then tool_push_dx cells more
    if tool_push_dx:
        xs = [tool.seg[i].left[0] for i in range(tool.num_seg)] + [tool.seg[i].right[0] for i in range(tool.num_seg)]
        if tool.has_fillet:
            xs.append(tool.fillet.p[0] + tool.fillet.r)
        gap = float(st["pos"][wp, 0].min()) - max(xs)
        t_push = (gap + tool_push_dx * dx) / tool.vel[0]
        mf.tool_translate(tool, t_push)
        st["pos"][~wp] += t_push * np.array([tool.vel[0], tool.vel[1]])
    st["tool"] = tool
    st["scene"] = sc
    return st


def load_product(mf, st, grid_kind=0, thermal_solver=0, jc_model=0, precision=0, flags=0, device=0):
    ctx = mf.Context(device)
    ctx.particles_create(st["pos"], st["vel"], st["rho"], st["h"], T=st["T"], fixed=st["fixed"],
                         tool_p=st["tool_p"], S=st["S"])
    for k in ("eps_pl", "eps_pl_dot", "fc", "ft", "n", "pos_t", "vel_t", "rho_t", "S_t", "T_t", "blanked"):
        ctx.set(k, st[k])
    bbmin, bbmax, h = st["grid"]
    ctx.grid_locked(grid_kind, bbmin, bbmax, h)
    ctx.set_constants(st["phys"], st["corr"], st["joco"], st["trml_wp"], st["trml_tool"])
    ctx.set_options(thermal_solver, jc_model, precision)
    ctx.set_flags(flags)
    ctx.tool_set(st["tool"])
    ctx.set_dt(st["dt"])
    return ctx


def load_oracle(orc, st, grid_kind=0, thermal_solver=0, jc_model=0):
    o = orc.Oracle(st["N"])
    for k in ("pos", "vel", "rho", "T", "h", "fixed", "S", "eps_pl", "eps_pl_dot", "fc", "ft", "n", "pos_t",
              "vel_t", "rho_t", "S_t", "T_t", "blanked"):
        o.set_field(k, st[k])
    o.set_field("tool_p", st["tool_p"])
    bbmin, bbmax, h = st["grid"]
    o.L.orc_set_grid_locked(o.s, grid_kind, bbmin[0], bbmin[1], bbmax[0], bbmax[1], h)
    phys = orc.OrcPhys(*[getattr(st["phys"], f) for f, _ in orc.OrcPhys._fields_])
    corr = orc.OrcCorr(*[getattr(st["corr"], f) for f, _ in orc.OrcCorr._fields_])
    joco = orc.OrcJoco(*[getattr(st["joco"], f) for f, _ in orc.OrcJoco._fields_])
    tw = orc.OrcTrml(*[getattr(st["trml_wp"], f) for f, _ in orc.OrcTrml._fields_])
    tt = orc.OrcTrml(*[getattr(st["trml_tool"], f) for f, _ in orc.OrcTrml._fields_])
    o.L.orc_set_constants(o.s, C.byref(phys), C.byref(corr), C.byref(joco), C.byref(tw), C.byref(tt))
    o.L.orc_set_options(o.s, thermal_solver, jc_model)
    o.L.orc_set_dt(o.s, st["dt"])
    tool = orc.OrcTool()
    C.memmove(C.byref(tool), C.byref(st["tool"]), C.sizeof(orc.OrcTool))
    o.L.orc_set_tool(o.s, C.byref(tool))
    o._keep = (phys, corr, joco, tw, tt, tool)
    return o


def product_tool_array(mf, t):
    return mf.tool_to_array(t)


def scene_state(mf, sc):
    """The state dict of an unperturbed scene (everything that is not set up starts at zero)."""
    s = sc.s
    N = sc.N
    st = {"N": N}
    for k in ("pos", "rho", "T", "h", "fixed", "tool_p"):
        st[k] = sc.array(k).copy()
    st["vel"] = np.zeros((N, 2))
    for k in ("eps_pl", "eps_pl_dot", "rho_t", "T_t", "blanked"):
        st[k] = np.zeros(N)
    for k in ("fc", "ft", "n", "pos_t", "vel_t"):
        st[k] = np.zeros((N, 2))
    for k in ("S", "S_t"):
        st[k] = np.zeros((N, 4))
    st["phys"], st["corr"], st["joco"] = s.phys, s.corr, s.joco
    st["trml_wp"], st["trml_tool"], st["dt"] = s.trml_wp, s.trml_tool, s.dt
    st["grid"] = (tuple(s.grid_bbmin), tuple(s.grid_bbmax), s.grid_h)
    tool = mf.ToolState()
    C.memmove(C.byref(tool), C.byref(s.tool), C.sizeof(mf.ToolState))
    st["tool"] = tool
    st["scene"] = sc
    return st
