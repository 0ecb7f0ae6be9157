"""Python access to the B200 SPH cutting step through its C ABI (``include/mfree_b200.h``).

The product is the native library ``lib/libmfree_b200.so`` (sm_100a CUDA + C++ host code);
this module only binds it with ctypes for the tests, the benchmark and interactive use.
There is no CPU fallback: without the library or without a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "libmfree_b200.so"

# ---- constants mirrored from include/mfree_b200.h ----
MF_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA runtime error", -3: "call out of order", -4: "size out of range",
          -5: "out of memory", -6: "no CUDA device", -7: "a kernel reported an internal error",
          -8: "state file input/output failed", -9: "state file failed its checks"}
MF_ERR_CORRUPT = -9
GRID_GREEN, GRID_ROTHLIN = 0, 1
THERMAL_BROOKSHAW, THERMAL_PSE = 0, 1
JC_JOHNSON_COOK, JC_TANH = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
OPT_KEEP_DERIVATIVES, OPT_NO_GRAPHS, OPT_SORT_EVERY_STEP, OPT_FUSED_PREDICTOR, OPT_NEIGHBOUR_LISTS = 1, 2, 4, 8, 16
BATCH_PHASES, BATCH_PERSISTENT = 0, 1
ERRF_BATCH_WAIT = 8  # mf_status.error_flags bit 3: a persistent batch launch's barrier wait expired

# name -> (field id, doubles per particle, is_int)
FIELDS = {
    "pos": (0, 2, False), "vel": (1, 2, False), "h": (2, 1, False), "rho": (3, 1, False), "p": (4, 1, False),
    "S": (5, 4, False), "R": (6, 4, False), "fc": (7, 2, False), "ft": (8, 2, False), "n": (9, 2, False),
    "fixed": (10, 1, False), "blanked": (11, 1, False), "tool_p": (12, 1, False), "eps_pl": (13, 1, False),
    "eps_pl_dot": (14, 1, False), "T": (15, 1, False), "pos_t": (16, 2, False), "vel_t": (17, 2, False),
    "rho_t": (18, 1, False), "S_t": (19, 4, False), "T_t": (20, 1, False), "S_der": (21, 4, False),
    "v_der": (22, 4, False), "idx": (23, 1, True), "hash": (24, 1, True), "id": (25, 1, True),
}


class MfError(RuntimeError):
    def __init__(self, code: int, where: str, cuda: int = 0):
        msg = f"{where}: {ERRORS.get(code, 'error')} ({code})"
        if cuda:
            msg += f", cudaError {cuda}"
        super().__init__(msg)
        self.code = code
        self.cuda = cuda


def _dfields(*names):
    return [(n, C.c_double) for n in names]


class Phys(C.Structure):
    _fields_ = _dfields("E", "nu", "rho0", "K", "G", "mass", "mass_tool")


class Trml(C.Structure):
    _fields_ = _dfields("cp", "tq", "k", "alpha", "T_init", "eta")


class Corr(C.Structure):
    _fields_ = _dfields("wdeltap", "stresseps", "xspheps", "alpha", "beta", "eta")


class Joco(C.Structure):
    _fields_ = _dfields("A", "B", "C", "n", "m", "Tmelt", "Tref", "eps_dot_ref", "tanh_a", "tanh_b", "tanh_c",
                        "tanh_d")


class Segment(C.Structure):
    _fields_ = [("left", C.c_double * 2), ("right", C.c_double * 2), ("a", C.c_double), ("b", C.c_double),
                ("vertical", C.c_int), ("n", C.c_double * 2)]


class Fillet(C.Structure):
    _fields_ = [("r", C.c_double), ("t1", C.c_double), ("t2", C.c_double), ("p", C.c_double * 2)]


class ToolState(C.Structure):
    _fields_ = [("num_seg", C.c_int), ("seg", Segment * 5), ("has_fillet", C.c_int), ("fillet", Fillet),
                ("mu", C.c_double), ("contact_alpha", C.c_double), ("slave_mass", C.c_double),
                ("vel", C.c_double * 2)]


class Status(C.Structure):
    _fields_ = [("steps", C.c_longlong), ("blanked", C.c_longlong), ("newly_blanked", C.c_longlong),
                ("out_of_grid", C.c_longlong), ("secant_cap_hits", C.c_longlong),
                ("max_cell_occupancy", C.c_int), ("error_flags", C.c_int), ("secant_iterations", C.c_longlong),
                ("sorts", C.c_longlong)]


_dp = C.POINTER(C.c_double)


class SceneStruct(C.Structure):
    _fields_ = [("N", C.c_int), ("n_workpiece", C.c_int), ("n_tool", C.c_int),
                ("pos", _dp), ("vel", _dp), ("rho", _dp), ("T", _dp), ("h", _dp), ("fixed", _dp), ("tool_p", _dp),
                ("phys", Phys), ("corr", Corr), ("joco", Joco), ("trml_wp", Trml), ("trml_tool", Trml),
                ("has_joco", C.c_int), ("tool", ToolState), ("grid_bbmin", C.c_double * 2),
                ("grid_bbmax", C.c_double * 2), ("grid_h", C.c_double), ("dt", C.c_double), ("t_final", C.c_double),
                ("feed", C.c_double), ("speed", C.c_double), ("grid_max_cell", C.c_int)]


class CutParams(C.Structure):
    _fields_ = ([("ny", C.c_int), ("nx_lattice", C.c_int)] +
                _dfields("dx", "lo_x", "lo_y", "hi_x", "hi_y", "hdx", "jitter") + [("seed", C.c_ulonglong)] +
                _dfields("rake", "clear", "chamfer", "speed", "feed", "mu_fric", "contact_alpha", "tool_tl_x",
                         "tool_tl_y", "tool_length", "tool_height", "tool_front_x") +
                [("sample_tool", C.c_int), ("use_thermals", C.c_int)] +
                _dfields("E", "nu", "rho0", "rho_tool") +
                [("joco", Joco), ("trml_wp", Trml), ("trml_tool", Trml), ("corr", Corr)] +
                _dfields("cfl", "cutting_distance"))


_lib = None


def lib():
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"native library missing: {LIB_PATH} (run mfree_iwf-ul_cut_gpu_b200/build.py)")
    L = C.CDLL(str(LIB_PATH))
    vp, i, d, ip = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_int)
    sig = {
        "mf_version": ([], i), "mf_error_string": ([i], C.c_char_p), "mf_last_cuda_error": ([vp], i),
        "mf_ctx_create": ([i, C.POINTER(vp)], i), "mf_ctx_destroy": ([vp], i),
        "mf_ctx_stream": ([vp, C.POINTER(vp)], i), "mf_set_flags": ([vp, i], i), "mf_set_neighbour_skin": ([vp, C.c_double], i),
        "mf_list_check": ([vp, vp, vp, vp], i), "mf_synchronize": ([vp], i),
        "mf_particles_create": ([vp, i] + [vp] * 8, i), "mf_particles_count": ([vp, ip], i),
        "mf_get_field": ([vp, i, vp], i), "mf_set_field": ([vp, i, vp], i),
        "mf_grid_create_locked": ([vp, i, d, d, d, d, d], i), "mf_grid_create_adaptive": ([vp, i, i], i),
        "mf_grid_geometry": ([vp, ip, ip, ip, vp], i), "mf_grid_build": ([vp], i),
        "mf_grid_get_cells": ([vp, vp, vp], i),
        "mf_set_constants": ([vp, C.POINTER(Phys), C.POINTER(Corr), C.POINTER(Joco), C.POINTER(Trml),
                              C.POINTER(Trml)], i),
        "mf_set_options": ([vp, i, i, i], i), "mf_set_dt": ([vp, d], i),
        "mf_set_contact_conductance": ([vp, d, d], i),
        "mf_tool_set": ([vp, C.POINTER(ToolState)], i), "mf_tool_get": ([vp, C.POINTER(ToolState)], i),
        "mf_step": ([vp, i], i), "mf_step_timed": ([vp, vp], i), "mf_step_stage": ([vp, i], i), "mf_report_force": ([vp, vp], i),
        "mf_tangent_mean_force": ([vp, i, i, i, vp, vp], i),
        "mf_tangent_mean_force_all": ([vp, i, i, vp, vp], i),
        "mf_tool_wear_usui": ([vp, d, d, vp], i), "mf_vtk_write_particles_async": ([vp, C.c_char_p], i),
        "mf_state_save": ([vp, C.c_char_p], i), "mf_state_load": ([vp, C.c_char_p], i),
        "mf_get_field_device": ([vp, i, vp, vp], i), "mf_set_field_device": ([vp, i, vp, vp], i),
        "mf_vtk_flush": ([vp], i), "mf_vtk_write_particle_arrays": ([C.c_char_p, i] + [vp] * 10, i),
        "mf_graph_capture": ([vp, i, C.POINTER(vp)], i), "mf_graph_destroy": ([vp], i),
        "mf_batch_create": ([C.POINTER(vp), i, i, C.POINTER(vp)], i), "mf_batch_steps_per_launch": ([vp, ip], i), "mf_batch_config": ([vp, ip, ip, ip], i),
        "mf_batch_step": ([vp, i], i), "mf_batch_destroy": ([vp], i),
        "mf_batch_set_form": ([vp, i, i, i], i), "mf_batch_form": ([vp, ip, ip], i),
        "mf_batch_set_wait_limit": ([vp, d], i),
        "mf_get_constants": ([vp, C.POINTER(Phys), C.POINTER(Corr), C.POINTER(Joco), C.POINTER(Trml),
                              C.POINTER(Trml), ip], i),
        "mf_force_log": ([vp, vp, i, ip], i), "mf_force_last_async": ([vp, vp], i), "mf_status_get": ([vp, C.POINTER(Status)], i),
        "mf_cut_params_reference": ([C.POINTER(CutParams), i, d, d, d, d, d], i),
        "mf_scene_cut": ([C.POINTER(CutParams), C.POINTER(C.POINTER(SceneStruct))], i),
        "mf_scene_setup_ref_cut": ([i, d, d, d, d, d, C.POINTER(C.POINTER(SceneStruct))], i),
        "mf_scene_setup_rings": ([i, C.POINTER(C.POINTER(SceneStruct))], i),
        "mf_scene_setup_impact": ([i, C.POINTER(C.POINTER(SceneStruct))], i),
        "mf_scene_free": ([C.POINTER(SceneStruct)], i),
        "mf_scene_upload": ([vp, C.POINTER(SceneStruct), i], i),
        "mf_tool_construct": ([d] * 8 + [C.POINTER(ToolState)], i),
        "mf_tool_sample": ([C.POINTER(ToolState), d, vp, i, ip], i),
        "mf_tool_translate": ([C.POINTER(ToolState), d], i),
        "mf_vtk_write_particles": ([vp, C.c_char_p], i), "mf_vtk_write_tool": ([C.POINTER(ToolState), C.c_char_p], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _as(a, n, w=1):
    if a is None:
        return None
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if a.size != n * w:
        raise ValueError(f"expected {n * w} values, got {a.size}")
    return a


class Scene:
    """A host scene (mf_scene): particle arrays, constants, tool, grid box and dt."""

    def __init__(self, ptr):
        self._p = ptr
        self.s = ptr.contents

    @classmethod
    def ref_cut(cls, ny=30, rake=10.0, clear=8.0, chamfer=0.002, speed=83.333328e-5 / 500.0 * 70.0, feed=0.01):
        """setup_ref_cut(ny, rake, clear, chamfer, speed, feed) (benchmarks.cpp:255-537)."""
        out = C.POINTER(SceneStruct)()
        rc = lib().mf_scene_setup_ref_cut(ny, rake, clear, chamfer, speed, feed, C.byref(out))
        if rc != MF_OK:
            raise MfError(rc, "mf_scene_setup_ref_cut")
        return cls(out)

    @classmethod
    def rings(cls, nbox):
        """setup_rings(nbox) (benchmarks.cpp:161-253): two colliding rubber-like rings."""
        out = C.POINTER(SceneStruct)()
        rc = lib().mf_scene_setup_rings(int(nbox), C.byref(out))
        if rc != MF_OK:
            raise MfError(rc, "mf_scene_setup_rings")
        return cls(out)

    @classmethod
    def impact(cls, nbox):
        """setup_impact(nbox) (benchmarks.cpp:23-159): a steel disc against a fixed wall."""
        out = C.POINTER(SceneStruct)()
        rc = lib().mf_scene_setup_impact(int(nbox), C.byref(out))
        if rc != MF_OK:
            raise MfError(rc, "mf_scene_setup_impact")
        return cls(out)

    @classmethod
    def from_params(cls, params: CutParams):
        out = C.POINTER(SceneStruct)()
        rc = lib().mf_scene_cut(C.byref(params), C.byref(out))
        if rc != MF_OK:
            raise MfError(rc, "mf_scene_cut")
        return cls(out)

    def __del__(self):
        try:
            if self._p:
                lib().mf_scene_free(self._p)
                self._p = None
        except Exception:
            pass

    @property
    def N(self):
        return self.s.N

    def array(self, name):
        w = 2 if name in ("pos", "vel") else 1
        p = getattr(self.s, name)
        return np.ctypeslib.as_array(p, shape=(self.s.N * w,)).reshape((self.s.N, w) if w > 1 else (self.s.N,))


def reference_cut_params(ny=30, rake=10.0, clear=8.0, chamfer=0.002, speed=83.333328e-5 / 500.0 * 70.0, feed=0.01):
    p = CutParams()
    rc = lib().mf_cut_params_reference(C.byref(p), ny, rake, clear, chamfer, speed, feed)
    if rc != MF_OK:
        raise MfError(rc, "mf_cut_params_reference")
    return p


class Context:
    """One particle system on one GPU (mf_ctx)."""

    def __init__(self, device: int = 0):
        self.L = lib()
        self.h = C.c_void_p()
        self._check(self.L.mf_ctx_create(device, C.byref(self.h)), "mf_ctx_create", ctx=False)

    def _check(self, rc, where, ctx=True):
        if rc != MF_OK:
            cuda = self.L.mf_last_cuda_error(self.h) if ctx and self.h else 0
            raise MfError(rc, where, cuda)

    def close(self):
        if self.h:
            self.L.mf_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # particles -----------------------------------------------------------------------
    def particles_create(self, pos, vel, rho, h, T=None, fixed=None, tool_p=None, S=None):
        n = int(np.asarray(rho).size)
        args = [_as(pos, n, 2), _as(vel, n, 2), _as(rho, n), _as(T, n), _as(h, n), _as(fixed, n), _as(tool_p, n),
                _as(S, n, 4)]
        self._keep = args
        self._check(self.L.mf_particles_create(self.h, n, *[_ptr(a) for a in args]), "mf_particles_create")
        self.N = n

    def get(self, name):
        fid, w, is_int = FIELDS[name]
        out = np.zeros(self.N * w, dtype=np.int32 if is_int else np.float64)
        self._check(self.L.mf_get_field(self.h, fid, _ptr(out)), f"mf_get_field({name})")
        return out.reshape(self.N, w) if w > 1 else out

    def set(self, name, values):
        fid, w, is_int = FIELDS[name]
        a = np.ascontiguousarray(np.asarray(values, dtype=np.int32 if is_int else np.float64).reshape(-1))
        if a.size != self.N * w:
            raise ValueError(name)
        self._check(self.L.mf_set_field(self.h, fid, _ptr(a)), f"mf_set_field({name})")

    # grid --------------------------------------------------------------------------------
    def grid_locked(self, kind, bbmin, bbmax, h):
        self._check(self.L.mf_grid_create_locked(self.h, kind, bbmin[0], bbmin[1], bbmax[0], bbmax[1], h),
                    "mf_grid_create_locked")

    def grid_adaptive(self, kind, max_cell):
        self._check(self.L.mf_grid_create_adaptive(self.h, kind, max_cell), "mf_grid_create_adaptive")

    def geometry(self):
        nx, ny, nc = C.c_int(), C.c_int(), C.c_int()
        d5 = np.zeros(5)
        self._check(self.L.mf_grid_geometry(self.h, C.byref(nx), C.byref(ny), C.byref(nc), _ptr(d5)),
                    "mf_grid_geometry")
        return {"nx": nx.value, "ny": ny.value, "num_cell": nc.value, "bbmin_x": d5[0], "bbmin_y": d5[1],
                "bbmax_x": d5[2], "bbmax_y": d5[3], "dx": d5[4]}

    def grid_build(self):
        self._check(self.L.mf_grid_build(self.h), "mf_grid_build")

    def cells(self):
        nc = self.geometry()["num_cell"]
        st = np.zeros(nc, dtype=np.int32)
        en = np.zeros(nc, dtype=np.int32)
        self._check(self.L.mf_grid_get_cells(self.h, _ptr(st), _ptr(en)), "mf_grid_get_cells")
        return st, en

    # constants / options ----------------------------------------------------------------
    def set_constants(self, phys, corr, joco=None, trml_wp=None, trml_tool=None):
        ref = lambda s: C.byref(s) if s is not None else None  # noqa: E731
        self._check(self.L.mf_set_constants(self.h, C.byref(phys), C.byref(corr), ref(joco), ref(trml_wp),
                                            ref(trml_tool)), "mf_set_constants")

    def state_save(self, path):
        self._check(self.L.mf_state_save(self.h, str(path).encode()), "mf_state_save")

    def state_load(self, path):
        self._check(self.L.mf_state_load(self.h, str(path).encode()), "mf_state_load")

    def get_device(self, name, device_ptr, stream=None):
        """Copy a field into device memory at `device_ptr` (an int address), on `stream`."""
        fid = FIELDS[name][0]
        self._check(self.L.mf_get_field_device(self.h, fid, C.c_void_p(device_ptr), C.c_void_p(stream)),
                    f"mf_get_field_device({name})")

    def set_device(self, name, device_ptr, stream=None):
        fid = FIELDS[name][0]
        self._check(self.L.mf_set_field_device(self.h, fid, C.c_void_p(device_ptr), C.c_void_p(stream)),
                    f"mf_set_field_device({name})")

    def tool_wear_usui(self, K, alpha):
        """(min, max, mean) Usui wear rate over the particles in contact (mf_tool_wear_usui)."""
        out = np.zeros(3)
        self._check(self.L.mf_tool_wear_usui(self.h, float(K), float(alpha), _ptr(out)), "mf_tool_wear_usui")
        return out

    def vtk_write_async(self, path):
        self._check(self.L.mf_vtk_write_particles_async(self.h, str(path).encode()), "mf_vtk_write_particles_async")

    def vtk_flush(self):
        self._check(self.L.mf_vtk_flush(self.h), "mf_vtk_flush")

    def get_constants(self):
        """(phys, corr, joco or None, trml_wp, trml_tool) as last set."""
        phys, corr, joco, tw, tt, hj = Phys(), Corr(), Joco(), Trml(), Trml(), C.c_int()
        self._check(self.L.mf_get_constants(self.h, C.byref(phys), C.byref(corr), C.byref(joco), C.byref(tw),
                                            C.byref(tt), C.byref(hj)), "mf_get_constants")
        return phys, corr, (joco if hj.value else None), tw, tt

    def tangent_mean_force(self, skip_steps, window_steps, param=-1):
        """Mean (Fc, Ff) over `window_steps` steps after `skip_steps`, from the current state, and
        its derivative with respect to parameter `param` (0..5: JC A, B, n, C, m, friction mu;
        -1: none). The state of the context is not changed (mf_tangent_mean_force)."""
        mean = np.zeros(2)
        dmean = np.zeros(2)
        self._check(self.L.mf_tangent_mean_force(self.h, int(skip_steps), int(window_steps), int(param), _ptr(mean),
                                                 _ptr(dmean)), "mf_tangent_mean_force")
        return mean, dmean

    def tangent_mean_force_all(self, skip_steps, window_steps):
        """Mean (Fc, Ff) as tangent_mean_force, with its derivatives with respect to all six
        parameters from one pass: row k of the (6, 2) array is d(mean Fc, mean Ff) / d(A, B, n,
        C, m, mu)[k] (mf_tangent_mean_force_all)."""
        mean = np.zeros(2)
        dmean = np.zeros(12)
        self._check(self.L.mf_tangent_mean_force_all(self.h, int(skip_steps), int(window_steps), _ptr(mean),
                                                     _ptr(dmean)), "mf_tangent_mean_force_all")
        return mean, dmean.reshape(6, 2)

    def set_options(self, thermal_solver=THERMAL_BROOKSHAW, jc_model=JC_JOHNSON_COOK, precision=PRECISION_FP64):
        self._check(self.L.mf_set_options(self.h, thermal_solver, jc_model, precision), "mf_set_options")

    def set_flags(self, flags):
        self._check(self.L.mf_set_flags(self.h, flags), "mf_set_flags")

    def set_neighbour_skin(self, skin):
        """Mixed form: skin of the neighbour lists (<= 0: a tenth of the cell size)."""
        self._check(self.L.mf_set_neighbour_skin(self.h, float(skin)), "mf_set_neighbour_skin")

    def list_check(self):
        """After a step on neighbour lists: the in-support pairs of the current pair records, how
        many of them the lists miss, and whether the records are already those of a next step
        that sorts (then the lists need not hold for them) (mf_list_check; O(N^2))."""
        pairs, missing, stale = C.c_longlong(), C.c_longlong(), C.c_int()
        self._check(self.L.mf_list_check(self.h, C.byref(pairs), C.byref(missing), C.byref(stale)),
                    "mf_list_check")
        return {"pairs": pairs.value, "missing": missing.value, "stale": bool(stale.value)}

    def set_dt(self, dt):
        self._check(self.L.mf_set_dt(self.h, dt), "mf_set_dt")

    def set_contact_conductance(self, h_contact, T_tool):
        """Tool-workpiece contact conductance (no reference counterpart; 0 = off)."""
        self._check(self.L.mf_set_contact_conductance(self.h, float(h_contact), float(T_tool)),
                    "mf_set_contact_conductance")

    def tool_set(self, tool: ToolState | None):
        self._check(self.L.mf_tool_set(self.h, C.byref(tool) if tool is not None else None), "mf_tool_set")

    def tool_get(self) -> ToolState:
        t = ToolState()
        self._check(self.L.mf_tool_get(self.h, C.byref(t)), "mf_tool_get")
        return t

    def upload_scene(self, scene: Scene, grid_kind=GRID_GREEN):
        self._check(self.L.mf_scene_upload(self.h, scene._p, grid_kind), "mf_scene_upload")
        self.N = scene.N

    # stepping ----------------------------------------------------------------------------
    def step(self, n=1):
        self._check(self.L.mf_step(self.h, n), "mf_step")

    def step_timed(self):
        """One step kernel by kernel; the device time (ms) of its four parts: cell sort,
        predictor, interactions + rates, corrector .. plasticity."""
        out = (C.c_float * 4)()
        self._check(self.L.mf_step_timed(self.h, C.cast(out, C.c_void_p)), "mf_step_timed")
        return np.array(out[:], dtype=np.float64)

    def stage(self, k):
        self._check(self.L.mf_step_stage(self.h, k), "mf_step_stage")

    def synchronize(self):
        self._check(self.L.mf_synchronize(self.h), "mf_synchronize")

    def report_force(self):
        out = np.zeros(2)
        self._check(self.L.mf_report_force(self.h, _ptr(out)), "mf_report_force")
        return out

    def force_last_async(self, host_ptr: int):
        """Queue a copy of the last step's force (2 doubles) to host memory at host_ptr."""
        self._check(self.L.mf_force_last_async(self.h, C.c_void_p(host_ptr)), "mf_force_last_async")

    def force_log(self, max_entries=1 << 16):
        out = np.zeros(2 * max_entries)
        n = C.c_int()
        self._check(self.L.mf_force_log(self.h, _ptr(out), max_entries, C.byref(n)), "mf_force_log")
        return out[: 2 * n.value].reshape(n.value, 2)

    def status(self) -> dict:
        s = Status()
        self._check(self.L.mf_status_get(self.h, C.byref(s)), "mf_status_get")
        return {k: getattr(s, k) for k, _ in Status._fields_}

    def stream(self) -> int:
        p = C.c_void_p()
        self._check(self.L.mf_ctx_stream(self.h, C.byref(p)), "mf_ctx_stream")
        return p.value or 0

    def vtk_write(self, path):
        self._check(self.L.mf_vtk_write_particles(self.h, str(path).encode()), "mf_vtk_write_particles")


class Batch:
    """Several contexts on one device advanced together by one graph launch (mf_batch_*).
    steps_per_launch = 0 lets the batch pick it by measuring a few launches."""

    def __init__(self, contexts, steps_per_launch=0):
        self.L = lib()
        self.contexts = list(contexts)
        arr = (C.c_void_p * len(self.contexts))(*[c.h for c in self.contexts])
        self.h = C.c_void_p()
        rc = self.L.mf_batch_create(arr, len(self.contexts), int(steps_per_launch), C.byref(self.h))
        if rc != MF_OK:
            raise MfError(rc, "mf_batch_create")
        self._read_config()

    def _read_config(self):
        k, fused, bs, form, bps = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self.L.mf_batch_config(self.h, C.byref(fused), C.byref(bs), C.byref(k))
        self.L.mf_batch_form(self.h, C.byref(form), C.byref(bps))
        self.steps_per_launch = k.value
        self.fused = bool(fused.value)  # batched kernels over all instances
        self.pair_block = bs.value
        self.form = form.value  # BATCH_PHASES: a launch per phase; BATCH_PERSISTENT: one per K steps
        self.blocks_per_sm = bps.value  # of the persistent form

    def set_form(self, form, blocks_per_sm=0, steps_per_launch=4):
        rc = self.L.mf_batch_set_form(self.h, int(form), int(blocks_per_sm), int(steps_per_launch))
        if rc != MF_OK:
            raise MfError(rc, "mf_batch_set_form")
        self._read_config()

    def set_wait_limit(self, seconds):
        rc = self.L.mf_batch_set_wait_limit(self.h, float(seconds))
        if rc != MF_OK:
            raise MfError(rc, "mf_batch_set_wait_limit")

    def step(self, n_launches=1):
        rc = self.L.mf_batch_step(self.h, int(n_launches))
        if rc != MF_OK:
            raise MfError(rc, "mf_batch_step")

    def close(self):
        if self.h:
            self.L.mf_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def probe_fp64(device=0) -> dict:
    """FP64 FMA throughput (TFLOP/s) and the latency (SM cycles) of a dependent double pow,
    log and division on `device` (mf_probe_fp64 of the benchmark-only lib/libmf_probe.so)."""
    path = LIB_PATH.parent / "libmf_probe.so"
    if not path.exists():
        raise RuntimeError(f"probe library missing: {path} (run mfree_iwf-ul_cut_gpu_b200/build.py)")
    probe = C.CDLL(str(path))
    probe.mf_probe_fp64.argtypes = [C.c_int] + [C.c_void_p] * 5
    probe.mf_probe_fp64.restype = C.c_int
    v = [C.c_double() for _ in range(5)]
    rc = probe.mf_probe_fp64(device, *[C.byref(x) for x in v])
    if rc != MF_OK:
        raise MfError(rc, "mf_probe_fp64")
    return {"fma_tflops": v[0].value, "pow_cycles": v[1].value, "log_cycles": v[2].value,
            "div_cycles": v[3].value, "sm_clock_mhz": v[4].value}


def tool_construct(tl, length, height, rake, clear, r, mu) -> ToolState:
    t = ToolState()
    rc = lib().mf_tool_construct(tl[0], tl[1], length, height, rake, clear, r, mu, C.byref(t))
    if rc != MF_OK:
        raise MfError(rc, "mf_tool_construct")
    return t


def tool_sample(tool: ToolState, dx: float) -> np.ndarray:
    n = C.c_int()
    lib().mf_tool_sample(C.byref(tool), dx, None, 0, C.byref(n))
    out = np.zeros(2 * n.value)
    rc = lib().mf_tool_sample(C.byref(tool), dx, _ptr(out), n.value, C.byref(n))
    if rc != MF_OK:
        raise MfError(rc, "mf_tool_sample")
    return out.reshape(-1, 2)


def vtk_write_particle_arrays(path, fields: dict) -> None:
    """The particle VTK file from host arrays: pos, vel, rho, p, T, eps_pl, S, fixed, blanked,
    tool_p (mf_vtk_write_particle_arrays)."""
    keys = ("pos", "vel", "rho", "p", "T", "eps_pl", "S", "fixed", "blanked", "tool_p")
    arrs = [np.ascontiguousarray(fields[k], dtype=np.float64) for k in keys]
    n = len(arrs[2])
    rc = lib().mf_vtk_write_particle_arrays(str(path).encode(), n, *[_ptr(a) for a in arrs])
    if rc != MF_OK:
        raise MfError(rc, "mf_vtk_write_particle_arrays")


def vtk_write_tool(tool: ToolState, path) -> None:
    """vtk_writer_write(const tool*, int) (mf_vtk_write_tool): the tool as triangles."""
    rc = lib().mf_vtk_write_tool(C.byref(tool), str(path).encode())
    if rc != MF_OK:
        raise MfError(rc, "mf_vtk_write_tool")


def tool_translate(tool: ToolState, dt: float) -> None:
    rc = lib().mf_tool_translate(C.byref(tool), dt)
    if rc != MF_OK:
        raise MfError(rc, "mf_tool_translate")


def tool_to_array(t: ToolState) -> dict:
    """Segments as an (n, 11) array in the oracle/_ref harness layout, plus fillet and misc."""
    seg = np.zeros((t.num_seg, 11))
    for i in range(t.num_seg):
        s = t.seg[i]
        seg[i] = [s.left[0], s.left[1], s.right[0], s.right[1], s.a, s.b, float(s.vertical), s.n[0], s.n[1], 0, 0]
    fil = np.array([t.fillet.r, t.fillet.t1, t.fillet.t2, t.fillet.p[0], t.fillet.p[1]]) if t.has_fillet else \
        np.zeros(5)
    return {"seg": seg, "fillet": fil, "mu": t.mu, "vel": np.array([t.vel[0], t.vel[1]])}
