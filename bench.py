"""Benchmark: particle-steps/s of the explicit 2D SPH cutting step on B200.

Workload (one "step" = one leap-frog step of the whole particle system): the ~150k-particle
orthogonal cut with the Brookshaw thermal solver and thermal contact (tool particles):
Ti6Al4V workpiece 2.0 mm x 0.6 mm on a 714 x 214 lattice, dx = 2.8 um, seeded jitter
+-0.5% dx, h = 1.5 dx, rigid tool (rake 0, clearance 7 deg, edge radius 5 um, depth of cut
50 um, 70 m/min, mu = 0.35), CFL 0.3. Synthetic inputs, generated by the project's scene
setup (a generalisation of the reference's setup_ref_cut).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Both forms run: plain FP64 and mixed FP32/FP64; the headline value is the mixed form.
Each timed step is bracketed by CUDA events on the library's stream, with the L2 flushed
(256 MiB written) between timed steps. Under torchrun (N > 1) every rank steps its own
replica of the scene (replicas only: the step has no data-path exchange); the time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "mfree_iwf-ul_cut_gpu_b200"
METRIC = "particle-steps/s at ~150k particles w/ thermal contact: mixed vs FP64, same B200"
# canonical algorithmic bytes per particle-step: one read and one write of the 224 B of mutable
# FP64 state plus a 32 B read of the per-particle constants
ALGO_BYTES_PER_PARTICLE_STEP = 480.0
# ncu summary of the pair kernel on this workload; its "dram bytes per launch" line is the
# roofline's measured traffic
PAIR_PROFILE = "profiles/k_pair_mixed_list_cut714x214.txt"  # the headline form's pair kernel
FLUSH_BYTES = 256 << 20


def load_package():
    name = "mfree_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def cut_params(mf, nx=714, ny=214, dx=2.8e-4):
    """The ~150k-particle cut (dx 2.8 um, 714 x 214) with thermal contact."""
    p = mf.reference_cut_params()
    p.nx_lattice, p.ny, p.dx = nx, ny, dx
    p.lo_x, p.lo_y = 0.0, 0.0
    p.jitter, p.seed = 0.005, 1
    p.rake, p.clear, p.chamfer = 0.0, 7.0, 5e-4
    p.feed = 0.005
    p.speed = 70.0 * 100.0 / 60.0e6  # 70 m/min in cm/us
    p.mu_fric = 0.35
    p.tool_front_x = -0.1 * dx
    p.sample_tool = 1
    p.use_thermals = 1
    p.E, p.nu, p.rho0 = 1.1, 0.35, 4.43
    jc = p.joco
    jc.A, jc.B, jc.n, jc.C, jc.m = 0.01098, 0.01092, 0.93, 0.014, 1.1
    jc.eps_dot_ref, jc.Tref, jc.Tmelt = 1e-6, 300.0, 1878.0
    p.trml_wp.cp, p.trml_wp.k, p.trml_wp.tq, p.trml_wp.eta = 553e-8, 7.1e-13, 0.9, 0.9
    p.cfl = 0.3
    return p


# the thermal solver of the timed forms (Brookshaw; the ~500k-particle configuration uses PSE)
SOLVER = {"thermal": 0, "skin": 0.0}  # thermal solver; neighbour-list skin (length, 0: default)

WORKLOAD = {"workload": "orthogonal cut, Ti6Al4V 2.0 x 0.6 mm, 714x214 lattice dx=2.8um + sampled tool "
                        "particles, Brookshaw thermal solver, thermal contact",
            "lattice": [714, 214], "dx_um": 2.8, "thermal_solver": "brookshaw", "grid": "green (locked)"}


WORKLOAD_BY_CONFIG = {
    "c1": {"workload": "orthogonal cut, Ti6Al4V 2.0 x 0.6 mm, 143x43 lattice dx=14um, adiabatic, no tool particles",
           "lattice": [143, 43], "dx_um": 14.0, "thermal_solver": "none", "grid": "green (locked)"},
    "c2": dict(WORKLOAD),
    "c3": {"workload": "orthogonal cut, Ti6Al4V 2.0 x 0.6 mm, 1290x387 lattice dx=1.55um + sampled tool particles, "
                       "PSE thermal solver, thermal contact", "lattice": [1290, 387], "dx_um": 1.55,
           "thermal_solver": "pse", "grid": "green (locked)"},
}


def config_params(mf, name, lattice_scale=1.0):
    """The scene parameters and workload description of a named configuration:
    c1 = 143 x 43 lattice, dx = 14 um, adiabatic, no tool particles (~6k);
    c2 = 714 x 214, dx = 2.8 um, Brookshaw, thermal contact (~150k, the benchmark);
    c3 = 1290 x 387, dx = 1.55 um, PSE, thermal contact (~500k)."""
    if name == "c1":
        p = cut_params(mf, nx=143, ny=43, dx=1.4e-3)
        p.sample_tool, p.use_thermals = 0, 0
        return p, mf.THERMAL_BROOKSHAW, dict(WORKLOAD_BY_CONFIG["c1"])
    if name == "c3":
        p = cut_params(mf, nx=1290, ny=387, dx=1.55e-4)
        return p, mf.THERMAL_PSE, dict(WORKLOAD_BY_CONFIG["c3"])
    sc = lattice_scale
    p = cut_params(mf, nx=int(round(714 * sc)), ny=int(round(214 * sc)), dx=2.8e-4 / sc)
    return p, mf.THERMAL_BROOKSHAW, dict(WORKLOAD)


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Max of a per-rank float over all ranks (identity at world size 1)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, world: int, device=None) -> float:
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML read from a thread
    every 20 ms (reading only; nothing is set), else nvidia-smi every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.thread = None
        self.samples = []  # (sm_mhz, max_mhz, set of reason names)

    def _nvml_handle(self, nv):
        try:  # the CUDA device's own GPU, whatever the visible-device order
            import torch

            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.dev)

    def _poll(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not self.stop.wait(0.02):
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                continue
            self.samples.append((sm, mx, {k for k, b in bits.items() if r & b}))

    def __enter__(self):
        import threading

        try:
            import pynvml as nv

            nv.nvmlInit()
            h = self._nvml_handle(nv)
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.dev), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            for ln in out.splitlines():
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    self.samples.append((float(parts[1]), float(parts[2]),
                                         {nm for nm, v in zip(self.NAMES, parts[5:9]) if v.lower() == "active"}))
                except ValueError:
                    continue

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [x[0] for x in self.samples]
        reasons = set().union(*[x[2] for x in self.samples])
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(x[1] for x in self.samples),
                "sm_mhz_min": float(min(sm)), "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.thread is not None else "nvidia-smi"}


SORT_RATE_STEPS = 1000  # untimed steps over which the list form's sort rate is counted


def time_form(mf, torch, scene, precision, steps, warmup, device, state_in=None, flags=0,
              sort_rate_steps=SORT_RATE_STEPS):
    """Per-step CUDA-event times (ms) of mf_step(1) with the L2 flushed between steps, then
    a few steps run kernel by kernel (mf_step_timed, L2 flushed) for the device time of each
    part: cell sort, predictor, interactions + rates (the pair kernel), corrector ..
    plasticity. With neighbour lists (flags) also one step that sorts and rebuilds the lists,
    forced by a host write. With state_in the steps start from a saved state of the
    same scene instead of its initial state."""
    ctx = mf.Context(device)
    ctx.upload_scene(scene, mf.GRID_GREEN)
    ctx.set_options(SOLVER["thermal"], mf.JC_JOHNSON_COOK, precision)
    ctx.set_neighbour_skin(SOLVER["skin"])
    ctx.set_flags(flags)
    if state_in:
        load_state(mf, ctx, state_in)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=device)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    ctx.step(warmup)
    ctx.synchronize()
    sorts0 = ctx.status()["sorts"]
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()
            ev[k][0].record(stream)
            ctx.step(1)
            ev[k][1].record(stream)
    torch.cuda.synchronize(device)
    step_ms = np.array([a.elapsed_time(b) for a, b in ev])
    st = ctx.status()
    extra = {"sorts_in_timed_steps": int(st["sorts"] - sorts0),
             "steps_per_sort": (warmup + steps) / max(st["sorts"], 1)}
    # the same number of steps back to back, one event pair, no flush (as a run executes them;
    # a step's working set is about the L2's size, so this is reported beside, not instead)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        a.record(stream)
        ctx.step(steps)
        b.record(stream)
    torch.cuda.synchronize(device)
    extra["back_to_back_ms_per_step"] = a.elapsed_time(b) / steps
    if precision == mf.PRECISION_MIXED and flags & mf.OPT_NEIGHBOUR_LISTS:
        # the trajectory's sort rate over a window longer than the timed steps (untimed): the
        # sorting steps' extra time is amortised at this rate
        if sort_rate_steps > 0:
            ctx.step(sort_rate_steps)
        ctx.synchronize()
        n_run = warmup + 2 * steps + sort_rate_steps
        extra["steps_per_sort"] = n_run / max(ctx.status()["sorts"], 1)
        extra["sort_rate_window_steps"] = n_run
    stages = []
    with torch.cuda.stream(stream):
        for _ in range(max(5, min(20, steps // 4))):
            flush.zero_()
            torch.cuda.synchronize(device)
            stages.append(ctx.step_timed())
    stages = np.array(stages)
    extra["stage_ms_median"] = [float(x) for x in np.median(stages, axis=0)]
    if precision == mf.PRECISION_MIXED and flags & mf.OPT_NEIGHBOUR_LISTS:
        sort_ms = []
        with torch.cuda.stream(stream):
            for _ in range(3):
                ctx.set("T", ctx.get("T"))  # a host write: the next step sorts and rebuilds the lists
                flush.zero_()
                torch.cuda.synchronize(device)
                sort_ms.append(float(ctx.step_timed().sum()))
        extra["sort_step_ms"] = float(np.median(sort_ms))
    ctx.close()
    return step_ms, stages[:, 2], st, extra


E2E_FIELDS = ("pos", "vel", "h", "rho", "T", "fixed", "blanked", "tool_p", "S", "eps_pl", "eps_pl_dot", "fc", "ft",
              "n", "pos_t", "vel_t", "rho_t", "S_t", "T_t")


def e2e_form(mf, torch, scene, precision, steps, device, flags=0):
    """End to end through the C ABI with host buffers. Outside the timed region: context,
    device buffers and the step graphs (created once per run). Inside: the complete particle
    state copied in from pinned host memory (mf_set_field, all per-particle fields, in one
    consistent order), `steps` x (mf_step(1) + a copy of that step's tool force to pinned
    host memory), and the final state copied back to the host."""
    ctx = mf.Context(device)
    ctx.upload_scene(scene, mf.GRID_GREEN)
    ctx.set_options(SOLVER["thermal"], mf.JC_JOHNSON_COOK, precision)
    ctx.set_neighbour_skin(SOLVER["skin"])
    ctx.set_flags(flags)
    ctx.step(2)  # builds the graphs
    ctx.synchronize()
    n = scene.N
    init = {}
    for f in E2E_FIELDS:
        w = mf.FIELDS[f][1]
        if f in ("pos", "vel", "h", "rho", "T", "fixed", "tool_p"):
            src = scene.array(f)
        else:
            src = np.zeros((n, w) if w > 1 else n)
        init[f] = torch.from_numpy(np.ascontiguousarray(src, dtype=np.float64)).pin_memory()
    forces = torch.zeros((steps, 2), dtype=torch.float64).pin_memory()
    out_fields = ("pos", "vel", "S", "rho", "T", "eps_pl")
    t0 = time.perf_counter()
    for f, t in init.items():
        ctx.set(f, t.numpy())
    for k in range(steps):
        ctx.step(1)
        ctx.force_last_async(forces[k].data_ptr())
    ctx.synchronize()
    out = {f: ctx.get(f) for f in out_fields}
    t1 = time.perf_counter()
    h2d = sum(t.numel() * 8 for t in init.values())
    d2h = sum(v.nbytes for v in out.values())
    finite = bool(np.isfinite(forces.numpy()).all())
    ctx.close()
    return (t1 - t0), h2d, d2h, finite


STATE_FIELDS = ("pos", "vel", "h", "rho", "T", "S", "fc", "ft", "n", "fixed", "blanked", "tool_p", "eps_pl",
                "eps_pl_dot", "pos_t", "vel_t", "rho_t", "S_t", "T_t", "id")


def save_state(mf, ctx, path, steps):
    """The whole particle state (array order of the last sort) and the tool, to an .npz."""
    import ctypes as C

    d = {k: ctx.get(k) for k in STATE_FIELDS}
    t = ctx.tool_get()
    d["tool_bytes"] = np.frombuffer(C.string_at(C.byref(t), C.sizeof(t)), dtype=np.uint8).copy()
    d["steps"] = np.array([steps])
    np.savez(path, **d)


def load_state(mf, ctx, path):
    """Overwrite a context's particle state and tool with a saved one (same scene)."""
    import ctypes as C

    d = np.load(path)
    for k in STATE_FIELDS:
        ctx.set(k, d[k])
    t = mf.ToolState()
    C.memmove(C.byref(t), d["tool_bytes"].tobytes(), C.sizeof(t))
    ctx.tool_set(t)
    return int(d["steps"][0])


def run_form(mf, scene, precision, steps, device, torch=None, state_out=None, flags=0, list_check_every=0,
             list_check_late=(0, 0), stop_on_nonfinite=False):
    """`steps` steps of one form from the scene's initial state. Returns the per-step tool
    force (steps x 2), the end state ordered by particle number, the device time (s) and the
    status. With neighbour lists (flags) and list_check_every > 0, the lists are checked by brute
    force (mf_list_check) every that many steps, outside the timed chunks, and from step
    list_check_late[0] on every list_check_late[1] steps when that is > 0; the status then
    carries the checks."""
    ctx = mf.Context(device)
    ctx.upload_scene(scene, mf.GRID_GREEN)
    ctx.set_options(SOLVER["thermal"], mf.JC_JOHNSON_COOK, precision)
    ctx.set_neighbour_skin(SOLVER["skin"])
    ctx.set_flags(flags)
    checking = list_check_every > 0 and bool(flags & mf.OPT_NEIGHBOUR_LISTS)
    checks, timeline = [], []
    forces, left, secs = [], steps, 0.0
    chunk = 50_000  # below the device force log's 65,536 entries
    if checking:
        chunk = min(chunk, list_check_every)
    while left > 0:
        n = min(left, chunk)
        done = steps - left
        if checking and list_check_late[1] > 0:
            if done >= list_check_late[0]:
                n = min(n, list_check_late[1])
            elif done + n > list_check_late[0]:
                n = list_check_late[0] - done
        if torch is not None:
            stream = torch.cuda.ExternalStream(ctx.stream(), device=device)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ctx.step(n)
            b.record(stream)
            torch.cuda.synchronize(device)
            secs += a.elapsed_time(b) * 1e-3
        else:
            ctx.step(n)
        forces.append(ctx.force_log())
        left -= n
        st = ctx.status()
        if not timeline or st["blanked"] != timeline[-1][1] or st["secant_cap_hits"] != timeline[-1][2]:
            timeline.append((steps - left, int(st["blanked"]), int(st["secant_cap_hits"])))
        if stop_on_nonfinite and not np.isfinite(forces[-1]).all():
            break
        if checking:
            c = ctx.list_check()
            st = ctx.status()
            checks.append({"steps": steps - left, "pairs": c["pairs"], "missing": c["missing"], "stale": c["stale"],
                           "blanked": st["blanked"], "sorts": st["sorts"], "secant_cap_hits": st["secant_cap_hits"]})
    order = np.argsort(ctx.get("id"))
    state = {k: ctx.get(k)[order] for k in ("S", "p", "eps_pl", "T", "tool_p", "blanked", "pos")}
    status = ctx.status()
    # (steps done, blanked, capped secant solves) where either changed: when a run went wrong
    status["timeline"] = timeline
    if checking:
        valid = [c for c in checks if not c["stale"]]
        bad = [c["steps"] for c in valid if c["missing"] > 0]
        status["list_checks"] = {"every": list_check_every, "checked": len(valid),
                                 "missing_total": int(sum(c["missing"] for c in valid)),
                                 "first_step_missing": bad[0] if bad else None, "log": checks}
    if state_out:
        save_state(mf, ctx, state_out, steps)
    ctx.close()
    return np.concatenate(forces), state, secs, status


def von_mises(S, p):
    """The return map's von Mises stress of (S - p I) (actions_gpu.cu:240-251)."""
    cxx, cxy, cyy, czz = S[:, 0] - p, S[:, 1], S[:, 2] - p, S[:, 3] - p
    return np.sqrt(np.maximum(cxx * cxx + cyy * cyy + czz * czz - cxx * cyy - cxx * czz - cyy * czz
                              + 3.0 * cxy * cxy, 0.0))


def finite_prefix(forces):
    """Steps before the first step whose tool force is not finite (all steps if none)."""
    bad = np.flatnonzero(~np.isfinite(forces).all(axis=1))
    return int(bad[0]) if bad.size else len(forces)


def chip_summary(scene, st):
    """Peak temperature rise over the workpiece and plastic strain of the chip (workpiece
    particles above the initial uncut surface), blanked particles left out."""
    y_top = scene.array("pos")[scene.array("tool_p") == 0.0, 1].max()
    wp = (st["tool_p"] == 0.0) & (st["blanked"] == 0.0)
    chip = wp & (st["pos"][:, 1] > y_top)
    T0 = scene.s.trml_wp.T_init
    return {"dT_peak": float(st["T"][wp].max() - T0),
            "eps_chip_max": float(st["eps_pl"][chip].max()) if chip.any() else 0.0,
            "eps_chip_mean": float(st["eps_pl"][chip].mean()) if chip.any() else 0.0,
            "n_chip": int(chip.sum())}


def form_errors(scene, ref, test):
    """Mixed (test) against FP64 (ref): relative error of the mean tool force over the steps
    both forms' forces are finite (all of them in a clean run), of the peak temperature rise and
    the chip's plastic strain, and relative L2 errors of the end fields over the workpiece
    particles blanked in neither."""
    (f64, s64), (fm, sm) = ref, test
    n = min(finite_prefix(f64), finite_prefix(fm))
    mask = (s64["tool_p"] == 0.0) & (s64["blanked"] == 0.0) & (sm["blanked"] == 0.0)
    c64, cm = chip_summary(scene, s64), chip_summary(scene, sm)

    def rel(a, b):
        return abs(a - b) / abs(b) if b else None

    def rel_l2(a, b):
        den = float(np.linalg.norm(b))
        return float(np.linalg.norm(a - b)) / den if den > 0 else float(np.linalg.norm(a - b))

    T0 = scene.s.trml_wp.T_init
    mean64, meanm = f64[:n].mean(axis=0), fm[:n].mean(axis=0)
    return {
        "force_steps": n,
        "first_nonfinite_force_step": {"fp64": finite_prefix(f64) if finite_prefix(f64) < len(f64) else None,
                                       "test": finite_prefix(fm) if finite_prefix(fm) < len(fm) else None},
        "mean_fc": [float(meanm[0]), float(mean64[0])],
        "mean_ff": [float(meanm[1]), float(mean64[1])],
        "mean_fc_rel_err": abs(float(meanm[0] - mean64[0])) / abs(float(mean64[0])) if mean64[0] else None,
        "mean_ff_rel_err": abs(float(meanm[1] - mean64[1])) / abs(float(mean64[1])) if mean64[1] else None,
        "von_mises_rel_l2": rel_l2(von_mises(sm["S"], sm["p"])[mask], von_mises(s64["S"], s64["p"])[mask]),
        "eps_pl_rel_l2": rel_l2(sm["eps_pl"][mask], s64["eps_pl"][mask]),
        "T_rise_rel_l2": rel_l2(sm["T"][mask] - T0, s64["T"][mask] - T0),
        "blanked": [int((sm["blanked"] != 0).sum()), int((s64["blanked"] != 0).sum())],
        "chip": {"test": cm, "fp64": c64},
        "dT_peak_rel_err": rel(cm["dT_peak"], c64["dT_peak"]),
        "eps_chip_max_rel_err": rel(cm["eps_chip_max"], c64["eps_chip_max"]),
        "eps_chip_mean_rel_err": rel(cm["eps_chip_mean"], c64["eps_chip_mean"]),
    }


def steps_per_mm(scene, params):
    """Leap-frog steps for 1 mm of tool travel (speed in cm/us, dt in us)."""
    return 0.1 / (params.speed * scene.s.dt)


def accuracy(mf, scene, params, steps, device, flags=0):
    """Mixed (with option flags) against FP64 over the first `steps` steps of the cut, both from
    the same state."""
    f64, s64, _, _ = run_form(mf, scene, mf.PRECISION_FP64, steps, device)
    fm, sm, _, stm = run_form(mf, scene, mf.PRECISION_MIXED, steps, device, flags=flags)
    out = {"steps": steps, "tool_travel_um": steps * scene.s.dt * params.speed * 1e4,
           "against": "the FP64 form (single steps equal to the oracle to 1e-12) from the same initial state",
           "mixed_sorts": int(stm["sorts"]), "mixed_error_flags": int(stm["error_flags"])}
    out.update(form_errors(scene, (f64, s64), (fm, sm)))
    return out


# the forms by name: precision and option flags. "mixed" (the headline): FP32 pair sums on
# neighbour lists kept between cell-list sorts; "mixed_sorted": the same sums with the cell list
# sorted every step, as the FP64 form does; "mixed_lists_fused": lists with the next step's
# predictor run in the finish kernel (measured slower; profiling only)
FORMS = {"fp64": ("PRECISION_FP64", ()), "mixed": ("PRECISION_MIXED", ("OPT_NEIGHBOUR_LISTS",)),
         "mixed_sorted": ("PRECISION_MIXED", ("OPT_SORT_EVERY_STEP",)),
         "mixed_lists_fused": ("PRECISION_MIXED", ("OPT_NEIGHBOUR_LISTS", "OPT_FUSED_PREDICTOR"))}
HEADLINE_FORMS = ("fp64", "mixed", "mixed_sorted")
CUT_FORMS = FORMS


def form_flags(mf, name):
    """Precision and option flags of a form; a name "<form>@p" is that form from initial
    positions moved by at most 1e-12 of the lattice spacing (cut runs only)."""
    flags = 0
    for f in FORMS[name.split("@")[0]][1]:
        flags |= getattr(mf, f)
    return getattr(mf, FORMS[name.split("@")[0]][0]), flags


def cut_together(mf, scene, params, mm, forms, device, out_dir, list_check_every=0, list_check_late=(0.0, 0),
                 state_out=None):
    """`mm` millimetres of cut in several forms at once, one context per form on its own
    stream, their steps launched in turns of 500 so that the forms' latency-bound kernels
    share the GPU (no per-form device time then); each form's run saved as cut_<form>.npz in
    out_dir (cut_compare reads them). A form whose tool force stops being finite is stopped
    at the end of that chunk; list checks as in run_form. With state_out, the FP64 form's end
    state is saved there (for --state-in)."""
    steps = int(round(mm * steps_per_mm(scene, params)))
    late = (int(round(list_check_late[0] * steps_per_mm(scene, params))), int(list_check_late[1]))
    runs = {}
    for form in forms:
        prec, flags = form_flags(mf, form)
        ctx = mf.Context(device)
        ctx.upload_scene(scene, mf.GRID_GREEN)
        ctx.set_options(SOLVER["thermal"], mf.JC_JOHNSON_COOK, prec)
        ctx.set_neighbour_skin(SOLVER["skin"])
        ctx.set_flags(flags)
        if form.endswith("@p"):  # a rounding-sized perturbation of the initial positions
            rng = np.random.default_rng(12345)
            pos = ctx.get("pos")
            ctx.set("pos", pos + (rng.random(pos.shape) - 0.5) * 2e-12 * params.dx)
        runs[form] = {"ctx": ctx, "forces": [], "timeline": [], "checks": [], "done": 0, "stopped": False,
                      "checking": list_check_every > 0 and bool(flags & mf.OPT_NEIGHBOUR_LISTS)}
    chunk = 20_000  # below the device force log's 65,536 entries
    if list_check_every > 0:
        chunk = min(chunk, list_check_every)
    t0 = time.time()
    while any(not r["stopped"] and r["done"] < steps for r in runs.values()):
        n = min(chunk, steps - min(r["done"] for r in runs.values() if not r["stopped"] and r["done"] < steps))
        if late[1] > 0:
            d = min(r["done"] for r in runs.values() if not r["stopped"] and r["done"] < steps)
            if d >= late[0]:
                n = min(n, late[1])
            elif d + n > late[0]:
                n = late[0] - d
        active = [r for r in runs.values() if not r["stopped"] and r["done"] < steps]
        for k0 in range(0, n, 500):
            for r in active:
                r["ctx"].step(min(500, n - k0))
        for r in active:
            ctx = r["ctx"]
            r["forces"].append(ctx.force_log())
            r["done"] += n
            st = ctx.status()
            tl = r["timeline"]
            if not tl or st["blanked"] != tl[-1][1] or st["secant_cap_hits"] != tl[-1][2]:
                tl.append((r["done"], int(st["blanked"]), int(st["secant_cap_hits"])))
            if r["checking"]:
                c = ctx.list_check()
                r["checks"].append({"steps": r["done"], "pairs": c["pairs"], "missing": c["missing"],
                                    "stale": c["stale"], "blanked": st["blanked"], "sorts": st["sorts"]})
            if not np.isfinite(r["forces"][-1]).all():
                r["stopped"] = True
    wall = time.time() - t0
    out = {}
    for form, r in runs.items():
        ctx = r["ctx"]
        if state_out and form == "fp64":
            save_state(mf, ctx, state_out, r["done"])
        order = np.argsort(ctx.get("id"))
        st = {k: ctx.get(k)[order] for k in ("S", "p", "eps_pl", "T", "tool_p", "blanked", "pos")}
        status = ctx.status()
        status["timeline"] = r["timeline"]
        if r["checking"]:
            valid = [c for c in r["checks"] if not c["stale"]]
            bad = [c["steps"] for c in valid if c["missing"] > 0]
            status["list_checks"] = {"every": list_check_every, "checked": len(valid),
                                     "missing_total": int(sum(c["missing"] for c in valid)),
                                     "first_step_missing": bad[0] if bad else None}
        ctx.close()
        f = np.concatenate(r["forces"])
        path = Path(out_dir) / f"cut_{form}.npz"
        np.savez(path, forces=f, secs=np.array([np.nan]), status=np.array([json.dumps(status)]),
                 steps_planned=np.array([steps]), **{"state_" + k: v for k, v in st.items()})
        out[form] = str(path)
    return out, wall


def cut_compare(mf, scene, paths):
    """Errors between the saved runs of cut_one: every form against the FP64 form (over the
    steps both forces are finite; end fields only where both runs reached the planned end)
    and the list forms against the sorted mixed form."""
    runs = {}
    for p in paths:
        d = np.load(p)
        st = {k[6:]: d[k] for k in d.files if k.startswith("state_")}
        status = json.loads(str(d["status"][0]))
        runs[Path(p).stem.replace("cut_", "")] = (d["forces"], st, float(d["secs"][0]), status,
                                                 int(d["steps_planned"][0]))
    out = {"forms": {}}
    blocks = 10  # mean force per tenth of the planned run, over its finite steps
    for name, (f, st, secs, status, planned) in runs.items():
        lc = status.get("list_checks")
        out["forms"][name] = {"steps": int(len(f)), "steps_planned": planned, "completed": len(f) == planned,
                              "first_nonfinite_force_step": finite_prefix(f) if finite_prefix(f) < len(f) else None,
                              "mean_force": f[:finite_prefix(f)].mean(axis=0).tolist(),
                              "block_mean_force": [f[k * planned // blocks:min((k + 1) * planned // blocks,
                                                                               finite_prefix(f))].mean(axis=0).tolist()
                                                   if k * planned // blocks < finite_prefix(f) else None
                                                   for k in range(blocks)],
                              "device_s": secs, "blanked": int(status["blanked"]),
                              "secant_cap_hits": int(status["secant_cap_hits"]), "sorts": int(status["sorts"]),
                              "timeline": status.get("timeline"), "chip": chip_summary(scene, st),
                              "list_checks": None if lc is None else {k: v for k, v in lc.items() if k != "log"}}

    def errs(ref, test):
        (fr, sr, _, _, pr), (ft, stt, _, _, pt) = runs[ref], runs[test]
        e = form_errors(scene, (fr, sr), (ft, stt))
        if not (len(fr) == pr and len(ft) == pt):  # a run stopped early: its end state is not the same instant
            for k in ("von_mises_rel_l2", "eps_pl_rel_l2", "T_rise_rel_l2", "chip", "dT_peak_rel_err",
                      "eps_chip_max_rel_err", "eps_chip_mean_rel_err"):
                e[k] = None
        return e

    for name in runs:
        if name != "fp64" and "fp64" in runs:
            out["forms"][name]["errors_against_fp64"] = errs("fp64", name)
        if name.endswith("@p") and name.split("@")[0] in runs:
            out["forms"][name]["errors_against_unperturbed"] = errs(name.split("@")[0], name)
        if name != "mixed_sorted" and name != "fp64" and "mixed_sorted" in runs:
            out["forms"][name]["errors_against_mixed_sorted"] = errs("mixed_sorted", name)
    return out


def sweep_params(mf, n_instances, seed=4):
    """The batched sweep: instances of the cut with N ~ U[3k, 40k] workpiece particles (dx
    scaled on the same 2.0 x 0.6 mm body), speed ~ U[30, 200] m/min, rake ~ U[-10, 15] deg,
    depth of cut ~ U[20, 100] um, JC A and B ~ U[0.9, 1.1] x the Ti6Al4V values."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_instances):
        n_wp = rng.uniform(3e3, 4e4)
        ny = max(8, int(round(np.sqrt(n_wp / (714.0 / 214.0)))))
        nx = int(round(ny * 714.0 / 214.0))
        p = cut_params(mf, nx=nx, ny=ny, dx=0.06 / ny)
        p.speed = rng.uniform(30.0, 200.0) * 100.0 / 60.0e6
        p.rake = rng.uniform(-10.0, 15.0)
        p.feed = rng.uniform(20e-4, 100e-4)
        p.joco.A *= rng.uniform(0.9, 1.1)
        p.joco.B *= rng.uniform(0.9, 1.1)
        out.append(p)
    return out


def batch_run(mf, torch, n_instances, steps, device):
    """The sweep stepped one instance at a time, all instances queued on their own streams,
    and as one batch (wall clock, host launch cost included)."""
    scenes = [mf.Scene.from_params(p) for p in sweep_params(mf, n_instances)]
    n_total = sum(sc.N for sc in scenes)

    def contexts():
        cs = []
        for sc in scenes:
            c = mf.Context(device)
            c.upload_scene(sc, mf.GRID_GREEN)
            c.set_options(mf.THERMAL_BROOKSHAW, mf.JC_JOHNSON_COOK, mf.PRECISION_MIXED)
            cs.append(c)
        return cs

    cs = contexts()
    for c in cs:
        c.step(4)  # graphs built, counts primed
    torch.cuda.synchronize(device)
    # one instance at a time, as a driver that owns one instance would run them
    t0 = time.perf_counter()
    for c in cs:
        c.step(steps)
        c.synchronize()
    one_s = time.perf_counter() - t0
    # all instances queued at once, each on its own stream (the GPU overlaps them)
    t0 = time.perf_counter()
    for c in cs:
        c.step(steps)
    for c in cs:
        c.synchronize()
    seq_s = time.perf_counter() - t0
    for c in cs:
        c.close()
    cs = contexts()
    b = mf.Batch(cs, steps_per_launch=0)
    k = b.steps_per_launch
    fused, pair_block = b.fused, b.pair_block
    form, bps = b.form, b.blocks_per_sm
    launches = max(1, steps // k)
    b.step(1)
    for c in cs:
        c.synchronize()
    t0 = time.perf_counter()
    b.step(launches)
    for c in cs:
        c.synchronize()
    bat_s = time.perf_counter() - t0
    # each launch form at a fixed setting, on the same (advancing) instances
    forms = {}
    if fused:
        for name, fm, fb, fk in (("phases_k16", mf.BATCH_PHASES, 0, 16), ("persistent_1_per_sm_k16", mf.BATCH_PERSISTENT, 1, 16),
                                 ("persistent_2_per_sm_k16", mf.BATCH_PERSISTENT, 2, 16)):
            try:
                b.set_form(fm, fb, fk)
            except mf.MfError as e:
                forms[name] = {"error": str(e)}
                continue
            nl = max(1, steps // fk)
            b.step(1)
            for c in cs:
                c.synchronize()
            t0 = time.perf_counter()
            b.step(nl)
            for c in cs:
                c.synchronize()
            w = time.perf_counter() - t0
            forms[name] = {"steps": nl * fk, "wall_s": w, "particle_steps_per_s": n_total * nl * fk / w,
                           "blocks_per_sm": b.blocks_per_sm}
    st = [c.status() for c in cs]
    b.close()
    for c in cs:
        c.close()
    return {"mode": "batch", "instances": n_instances, "particles_total": n_total,
            "particles_min_max": [min(sc.N for sc in scenes), max(sc.N for sc in scenes)],
            "precision": "mixed", "steps_per_launch": k, "batched_kernels": fused, "pair_block": pair_block,
            "form": ("persistent" if form == mf.BATCH_PERSISTENT else "phases"), "persistent_blocks_per_sm": bps,
            "launches_per_step": (f"one cooperative launch per {k} steps for all instances ({bps} blocks per SM)"
                                  if form == mf.BATCH_PERSISTENT else "one per step phase for all instances"
                                  if fused else "one child graph per instance"),
            "forms": forms,
            "one_at_a_time": {"steps": steps, "wall_s": one_s, "particle_steps_per_s": n_total * steps / one_s},
            "streams": {"steps": steps, "wall_s": seq_s, "particle_steps_per_s": n_total * steps / seq_s},
            "batched": {"steps": launches * k, "wall_s": bat_s,
                        "particle_steps_per_s": n_total * launches * k / bat_s},
            "batched_over_one_at_a_time": (launches * k / bat_s) / (steps / one_s),
            "batched_over_streams": (launches * k / bat_s) / (steps / seq_s),
            "blanked": sum(x["blanked"] for x in st), "error_flags": max(x["error_flags"] for x in st)}


REF_FUNCTIONS = ("the reference's own kernels.cuh / plasticity.cuh functions (cubic_spline, lapl_pse, "
                 "sigma_yield, solve_secant) compiled for the host, inside the C restatement's OpenMP loops over "
                 "the same cell lists")


def cpu_kind(orc, o):
    """Put oracle state `o` on the reference's host-compiled per-particle functions where they
    were built (cpu_baseline kind "reference"), else leave the restatement ("port")."""
    return "reference" if orc.use_reference_functions(o) else "port"


def cpu_baseline(mf, scene, seconds=12.0, max_steps=5000):
    """The CPU path (C, OpenMP, all host threads) on the same scene: bounded sample."""
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "tests"))
    import binding as orc
    import build_oracle
    from helpers import load_oracle

    build_oracle.build_oracle()
    st = scene_state(mf, scene)
    o = load_oracle(orc, st)
    kind = cpu_kind(orc, o)
    o.L.orc_step(o.s)  # warm-up (first-touch of the pages)
    t0 = time.perf_counter()
    o.L.orc_step(o.s)
    t1 = time.perf_counter() - t0
    k = int(max(1, min(max_steps, seconds / max(t1, 1e-6))))
    t0 = time.perf_counter()
    o.L.orc_steps(o.s, k)
    dt = time.perf_counter() - t0
    what = REF_FUNCTIONS if kind == "reference" else "the C restatement, OpenMP"
    return {"value": scene.N * k / dt, "unit": "particle-steps/s", "cores": int(orc.lib().orc_get_threads()),
            "kind": kind, "sample": f"{k} steps of the full {scene.N}-particle scene after 1 warm-up step "
                                    f"({what}), {dt:.1f} s"}


def reference_gpu_baseline(mf, scene, steps=200, warmup=10):
    """The reference's own FP64 CUDA build (its sources compiled unchanged for sm_100a with a
    shim for the removed texture-reference API, oracle/_ref/libref_gpu.so; Brookshaw, the
    build's solver) stepping the same scene on the same B200 through its leap_frog::step:
    `steps` steps back to back between CUDA events on its stream (no L2 flush: compare with
    the forms' back_to_back_ms_per_step). A reported baseline, not the product."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import ctypes as C

    import binding as orc

    if orc.ref_gpu() is None:
        return {"unavailable": "oracle/_ref/libref_gpu.so was not built (no reference tree where build() ran)"}
    if SOLVER["thermal"] != mf.THERMAL_BROOKSHAW:
        return {"unavailable": "the reference's build selects the Brookshaw solver in its types.h; this "
                               "configuration uses PSE"}
    st = scene_state(mf, scene)

    def doubles(struct):
        return [getattr(struct, f) for f, _ in struct._fields_]

    tool = orc.OrcTool()
    C.memmove(C.byref(tool), C.byref(st["tool"]), C.sizeof(orc.OrcTool))
    r = orc.RefGPU(st, doubles(st["phys"]), doubles(st["corr"]), doubles(st["joco"]), doubles(st["trml_wp"]),
                   doubles(st["trml_tool"]), tool)
    r.step(warmup)
    ms = r.run_timed(steps)
    return {"value": scene.N * steps / (ms * 1e-3), "unit": "particle-steps/s", "ms_per_step": ms / steps,
            "steps": steps, "warmup": warmup, "dtype": "f64",
            "what": "the reference's own FP64 CUDA step (leap_frog::step, unchanged sources + texture shim, "
                    "sm_100a), same scene, same GPU, steps back to back on its stream"}


def scene_state(mf, scene):
    """The scene as the state dict tests/helpers.load_oracle expects."""
    import ctypes as C

    s = scene.s
    N = scene.N
    st = {"N": N}
    for k in ("pos", "vel", "rho", "T", "h", "fixed", "tool_p"):
        st[k] = scene.array(k).copy()
    z1, z2, z4 = np.zeros(N), np.zeros((N, 2)), np.zeros((N, 4))
    st.update({"S": z4, "eps_pl": z1, "eps_pl_dot": z1, "fc": z2, "ft": z2, "n": z2, "pos_t": z2, "vel_t": z2,
               "rho_t": z1, "S_t": z4, "T_t": z1, "blanked": z1})
    st.update({"phys": s.phys, "corr": s.corr, "joco": s.joco, "trml_wp": s.trml_wp, "trml_tool": s.trml_tool,
               "dt": s.dt, "grid": (tuple(s.grid_bbmin), tuple(s.grid_bbmax), s.grid_h)})
    t = mf.ToolState()
    C.memmove(C.byref(t), C.byref(s.tool), C.sizeof(mf.ToolState))
    st["tool"] = t
    return st


def kernels_per_step(mf, precision):
    # locked grid, Brookshaw, JC plasticity: scan, scatter, reorder/predict, pair, finish (which
    # also hashes and counts the particles for the next step), return map of the plastic list
    return 6


def oracle_from_scene_file(orc, path):
    """An oracle state holding a scene file's initial scene (oracle/scene_file.py): the inputs of
    the reference arm, loaded without the product library."""
    import ctypes as C

    d = np.load(path)
    N = int(d["pos"].shape[0])
    o = orc.Oracle(N)
    for k in ("pos", "vel", "rho", "T", "h", "fixed", "tool_p"):
        o.set_field(k, d[k])
    g = d["grid"]
    o.L.orc_set_grid_locked(o.s, 0, g[0], g[1], g[2], g[3], g[4])
    phys = orc.OrcPhys(*d["phys"])
    corr = orc.OrcCorr(*d["corr"])
    joco = orc.OrcJoco(*d["joco"])
    tw, tt = orc.OrcTrml(*d["trml_wp"]), orc.OrcTrml(*d["trml_tool"])
    o.L.orc_set_constants(o.s, C.byref(phys), C.byref(corr), C.byref(joco), C.byref(tw), C.byref(tt))
    o.L.orc_set_options(o.s, int(d["thermal_solver"][0]), 0)
    o.L.orc_set_dt(o.s, float(d["dt"][0]))
    tool = orc.OrcTool()
    C.memmove(C.byref(tool), d["tool"].tobytes(), C.sizeof(orc.OrcTool))
    o.L.orc_set_tool(o.s, C.byref(tool))
    o._keep = (phys, corr, joco, tw, tt, tool)
    return o, N, int(d["n_tool"][0])


def run_reference(args):
    """--impl reference: the reference path's CPU implementation on the host cores (the
    reference's own per-particle functions inside the oracle's OpenMP loops where they were
    built, else the oracle's restatement), on the configuration's scene read from its scene
    file (oracle/scene_file.py), so that this arm never loads the product library."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import binding as orc
    import build_oracle
    import scene_file

    build_oracle.build_oracle()
    path = scene_file.scene_path(args.config)
    if not path.exists():
        print(json.dumps({"impl": "reference", "unavailable": f"scene file {path.name} missing: run "
                          f"python oracle/scene_file.py {args.config} (or __graft_entry__.build())"}), flush=True)
        return 0
    o, N, n_tool = oracle_from_scene_file(orc, path)
    kind = cpu_kind(orc, o)
    workload = dict(WORKLOAD_BY_CONFIG[args.config])
    # each "step" is one full oracle step; bound the run to a few minutes
    o.L.orc_step(o.s)
    t0 = time.perf_counter()
    o.L.orc_step(o.s)
    t1 = time.perf_counter() - t0
    budget = 150.0
    warm = min(args.warmup, max(0, int(budget * 0.2 / max(t1, 1e-6))))
    steps = max(1, min(args.steps, int(budget * 0.8 / max(t1, 1e-6))))
    for _ in range(warm):
        o.L.orc_step(o.s)
    t0 = time.perf_counter()
    o.L.orc_steps(o.s, steps)
    dt = time.perf_counter() - t0
    v = N * steps / dt
    cores = int(orc.lib().orc_get_threads())
    line = {"metric": METRIC, "value": v, "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": warm, "ms_per_step": dt / steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": dict(workload, name=args.config, n_particles=N, n_tool=n_tool,
                           scene=f"oracle/_build/scenes/{path.name}"),
            "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": cores, "kind": kind,
                             "sample": f"{steps} full steps of the {N}-particle scene (requested "
                                       f"{args.steps}), " + (REF_FUNCTIONS if kind == "reference" else
                                                             "C restatement of the reference step, OpenMP")},
            "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def profiled_traffic(path, n_particles):
    """DRAM bytes (read + write) per pair-kernel launch from the committed ncu summary of the
    same workload, or None when there is none for this particle count."""
    if not path.exists():
        return None
    text = path.read_text()
    if f"{n_particles} particles" not in text:
        return None
    for line in text.splitlines():
        if line.startswith("dram bytes per launch (read + write):"):
            return float(line.split(":", 1)[1].split()[0])
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sort-rate-steps", type=int, default=SORT_RATE_STEPS,
                    help="untimed steps over which the neighbour-list form's sort rate is counted")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched form's 64-instance sweep that the benchmark line carries")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own CUDA build on the same GPU (a reported baseline)")
    ap.add_argument("--e2e-steps", type=int, default=500)
    ap.add_argument("--accuracy-steps", type=int, default=20_000,
                    help="steps of the mixed-against-FP64 error report (0: off)")
    ap.add_argument("--cut-mm", type=float, default=0.0,
                    help="instead of the benchmark: run this many mm of cut in the --cut-forms (together on the "
                         "GPU, one context and stream each) and report each form's errors against the FP64 form")
    ap.add_argument("--cut-forms", default="fp64,mixed,mixed_sorted")
    ap.add_argument("--list-check-every", type=int, default=0,
                    help="with --cut-mm: check the list forms' neighbour lists by brute force (mf_list_check) every "
                         "this many steps (0: never)")
    ap.add_argument("--list-check-late", default="0,0",
                    help="with --list-check-every: 'MM,STEPS' = from MM mm of cut on, check every STEPS steps")
    ap.add_argument("--cut-dir", default="/tmp", help="with --cut-mm: where each form's run is saved (.npz)")
    ap.add_argument("--cut-compare", nargs="+", default=None,
                    help="instead of the benchmark: errors between runs saved by --cut-mm (cut_<form>.npz)")
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c3"],
                    help="c2 (default): the ~150k-particle cut with thermal contact, the benchmark; "
                         "c1: the ~6k adiabatic cut; c3: the ~500k cut with the PSE solver")
    ap.add_argument("--batch", type=int, default=0,
                    help="instead of the benchmark: the batched sweep of this many instances (mixed), "
                         "stepped one by one and as one batch")
    ap.add_argument("--state-out", default=None,
                    help="with --cut-mm: save the FP64 form's end state (.npz) for --state-in")
    ap.add_argument("--state-in", default=None,
                    help="time both forms from this saved state of the same scene (e.g. mid-cut) "
                         "instead of the initial state")
    ap.add_argument("--skin", type=float, default=0.0,
                    help="neighbour-list skin of the mixed form as a fraction of the cell size (0: the "
                         "library's default, a tenth)")
    ap.add_argument("--forms", default=",".join(HEADLINE_FORMS),
                    help="comma-separated forms to time (all three for the benchmark line; one, e.g. "
                         "'mixed', for a profiling run)")
    ap.add_argument("--lattice-scale", type=float, default=1.0,
                    help="lattice points per dimension relative to 714 x 214 (same 2.0 x 0.6 mm body); "
                         "values below 1 give the smaller profiling case")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)

    import torch

    world, rank, local = dist_env()
    device = local if world > 1 else 0
    torch.cuda.set_device(device)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", device))
    mf = load_package()
    sc = args.lattice_scale
    params, SOLVER["thermal"], workload = config_params(mf, args.config, sc)
    scene = mf.Scene.from_params(params)
    SOLVER["skin"] = args.skin * scene.s.grid_h
    N = scene.N
    if args.batch > 0:
        if rank == 0:
            print(json.dumps(batch_run(mf, torch, args.batch, args.steps, device)), flush=True)
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return 0
    if args.cut_compare:
        print(json.dumps(cut_compare(mf, scene, args.cut_compare)), flush=True)
        return 0
    if args.cut_mm > 0:
        if rank == 0:
            lmm, lst = args.list_check_late.split(",")
            paths, wall = cut_together(mf, scene, params, args.cut_mm, args.cut_forms.split(","), device,
                                       args.cut_dir, list_check_every=args.list_check_every,
                                       list_check_late=(float(lmm), int(lst)), state_out=args.state_out)
            res = cut_compare(mf, scene, list(paths.values()))
            res.update({"mode": "cut", "mm": args.cut_mm, "wall_s_all_forms": wall, "n_particles": N,
                        "steps_per_mm": steps_per_mm(scene, params)})
            print(json.dumps(res), flush=True)
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return 0

    results = {}
    forms = [(name,) + form_flags(mf, name) for name in FORMS if name in args.forms.split(",")]
    # one clock record over every form's timing (each form's own timed region lasts well under a
    # second, about the sampler's start-up time)
    with ClockSampler(device) as cs:
        for name, prec, flags in forms:
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize(device)
            step_ms, pair_ms, st, extra = time_form(mf, torch, scene, prec, args.steps, args.warmup, device,
                                                    args.state_in, flags, args.sort_rate_steps)
            total_ms = max_over_ranks(float(step_ms.sum()), world, device=f"cuda:{device}")
            results[name] = {"ms_per_step": total_ms / args.steps, "pair_kernel_ms": float(np.median(pair_ms)),
                             "status": st, **extra}
    clocks = cs.summary()
    if set(results) != set(HEADLINE_FORMS):  # a profiling run: no benchmark line
        if rank == 0:
            print(json.dumps({"forms": {f: {k: v for k, v in r.items() if k != "status"}
                                        for f, r in results.items()}}), flush=True)
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0
    acc = None
    if rank == 0 and args.accuracy_steps > 0:
        acc = accuracy(mf, scene, params, args.accuracy_steps, device, flags=form_flags(mf, "mixed")[1])
    # neighbour lists: the timed steps may hold fewer sorts than a run; charge each step its
    # share of a sorting step's extra time, at the context's steps per sort
    for ml in results.values():
        if "sort_step_ms" not in ml:
            continue
        ml["timed_ms_per_step"] = ml["ms_per_step"]
        if ml["sorts_in_timed_steps"] < args.steps:  # (without lists, e.g. PSE, every timed step sorted)
            ml["ms_per_step"] += max(0.0, ml["sort_step_ms"] - ml["timed_ms_per_step"]) / ml["steps_per_sort"]
    particles = sum_over_ranks(float(N), world, device=f"cuda:{device}")
    for name, r in results.items():
        r["value"] = particles / (r["ms_per_step"] * 1e-3)
    # roofline of the dominant kernel (the pair kernel) on the canonical per-particle bytes
    peaks_file = ROOT / "MEASURED_PEAKS.json"
    if peaks_file.exists():
        peak = float(json.loads(peaks_file.read_text())["hbm_gbs"])
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    for r in results.values():  # every form on the same canonical bytes: whole step, pair kernel
        r["roofline_frac_step"] = ALGO_BYTES_PER_PARTICLE_STEP * N / (r["ms_per_step"] * 1e-3) / 1e9 / peak
        r["roofline_frac_pair_kernel"] = (ALGO_BYTES_PER_PARTICLE_STEP * N / (r["pair_kernel_ms"] * 1e-3) / 1e9
                                          / peak)
    head = results["mixed"]
    achieved = ALGO_BYTES_PER_PARTICLE_STEP * N / (head["pair_kernel_ms"] * 1e-3) / 1e9
    step_achieved = ALGO_BYTES_PER_PARTICLE_STEP * N / (head["ms_per_step"] * 1e-3) / 1e9
    traffic = profiled_traffic(ROOT / PAIR_PROFILE, N) if args.lattice_scale == 1.0 else None

    e2e = e2e_fp64 = None
    if rank == 0:
        for prec in (mf.PRECISION_MIXED, mf.PRECISION_FP64):
            flags = form_flags(mf, "mixed")[1] if prec == mf.PRECISION_MIXED else 0
            secs, h2d, d2h, finite = e2e_form(mf, torch, scene, prec, args.e2e_steps, device, flags)
            if not finite:
                raise SystemExit("e2e: non-finite tool force in the end-to-end run")
            line_e2e = {"value": N * args.e2e_steps / secs, "unit": "particle-steps/s",
                        "h2d_bytes_per_step": h2d / args.e2e_steps, "d2h_bytes_per_step": 16 + d2h / args.e2e_steps,
                        "steps": args.e2e_steps,
                        "what": "state in from pinned host memory, per step mf_step(1) + tool force to pinned host "
                                "memory, final state out; wall clock"}
            if prec == mf.PRECISION_MIXED:
                e2e = line_e2e
            else:
                e2e_fp64 = dict(line_e2e, form="fp64")
    fp64_probe = mf.probe_fp64(device) if rank == 0 else None
    spm = steps_per_mm(scene, params)
    batched = None
    if rank == 0 and not args.no_batch:  # the batched form on the 64-instance parameter sweep
        batched = batch_run(mf, torch, 64, 64, device)
    cpu = ref_gpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(mf, scene)
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu_baseline(mf, scene)
        if "ms_per_step" in ref_gpu:
            ref_gpu["fp64_form_speedup_back_to_back"] = (ref_gpu["ms_per_step"]
                                                        / results["fp64"]["back_to_back_ms_per_step"])
            ref_gpu["mixed_form_speedup_back_to_back"] = (ref_gpu["ms_per_step"]
                                                         / results["mixed"]["back_to_back_ms_per_step"])
    if world > 1:
        torch.distributed.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": head["value"], "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 mixed",
            "data": "synthetic",
            "config": dict(workload, name=args.config, n_particles=N, n_workpiece=scene.s.n_workpiece,
                           n_tool=scene.s.n_tool,
                           start_state=(f"saved state {args.state_in}" if args.state_in else "initial scene"),
                           parallelism=f"replicas x{world}", l2="flushed between timed steps (256 MiB write)",
                           mixed_form="FP32 pair sums on neighbour lists (MF_OPT_NEIGHBOUR_LISTS), the cell list "
                                      "sorted when a particle moved 0.45 skin from its list's build position",
                           global_particles=N * world),
            "forms": dict(
                {f: {k: v for k, v in r.items() if k != "status"} for f, r in results.items()},
                mixed_over_fp64=results["mixed"]["value"] / results["fp64"]["value"],
                mixed_over_fp64_back_to_back=(results["fp64"]["back_to_back_ms_per_step"]
                                              / results["mixed"]["back_to_back_ms_per_step"]),
                mixed_sorted_over_fp64=results["mixed_sorted"]["value"] / results["fp64"]["value"],
                wall_s_per_mm_cut={f: r["ms_per_step"] * 1e-3 * spm for f, r in results.items()},
                steps_per_mm_cut=spm,
                note="mixed (the headline): FP32 pair sums on neighbour lists kept between cell-list sorts "
                     "(MF_OPT_NEIGHBOUR_LISTS; ms_per_step = timed steps + each step's share of a sorting step's "
                     "extra time at steps_per_sort, the sort rate counted over sort_rate_window_steps steps of the same "
                     "run, warm-up, timed and back-to-back steps included); mixed_sorted: the same sums with the cell list sorted every "
                     "step, as in the FP64 form; pair_kernel_ms: median "
                     "of steps launched kernel by kernel (mf_step_timed) after an L2 flush; "
                     "back_to_back_ms_per_step: the same number of steps without flushes, one event pair "
                     "(reported beside the flushed headline)"),
            "mixed_error": acc,
            "fp64_probe": fp64_probe,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "kernel": "k_pair_mixed<true> (neighbour lists)",
                         "algorithmic_bytes_per_particle": ALGO_BYTES_PER_PARTICLE_STEP,
                         "step_achieved": step_achieved, "step_frac": step_achieved / peak},
            "gpu_launches": kernels_per_step(mf, mf.PRECISION_MIXED) * args.steps,
            "clocks": clocks,
            "e2e": e2e,
            "e2e_fp64": e2e_fp64,
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "batched_sweep": batched,
            "status": {k: v for k, v in results["mixed"]["status"].items()},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
