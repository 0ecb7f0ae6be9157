"""ctypes bindings of the oracle (``liboracle.so``) and of the host-compiled reference
pieces (``oracle/_ref/libref_host.so``).

ORACLE - test infrastructure only: imported by ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg, never by the product.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libref_host.so"

# field ids (sph_oracle.h), same numbering as the product's MF_FIELD_*
FIELDS = {
    "pos": (0, 2), "vel": (1, 2), "h": (2, 1), "rho": (3, 1), "p": (4, 1), "S": (5, 4), "R": (6, 4),
    "fc": (7, 2), "ft": (8, 2), "n": (9, 2), "fixed": (10, 1), "blanked": (11, 1), "tool_p": (12, 1),
    "eps_pl": (13, 1), "eps_pl_dot": (14, 1), "T": (15, 1), "pos_t": (16, 2), "vel_t": (17, 2),
    "rho_t": (18, 1), "S_t": (19, 4), "T_t": (20, 1), "S_der": (21, 4), "v_der": (22, 4),
    "idx": (23, 1), "hash": (24, 1),
}
INT_FIELDS = ("idx", "hash")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OrcPhys(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("E", "nu", "rho0", "K", "G", "mass", "mass_tool")]


class OrcTrml(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("cp", "tq", "k", "alpha", "T_init", "eta")]


class OrcCorr(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("wdeltap", "stresseps", "xspheps", "alpha", "beta", "eta")]


class OrcJoco(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("A", "B", "C", "n", "m", "Tmelt", "Tref", "eps_dot_ref",
                                          "tanh_a", "tanh_b", "tanh_c", "tanh_d")]


class OrcSegment(C.Structure):
    _fields_ = [("left", C.c_double * 2), ("right", C.c_double * 2), ("a", C.c_double), ("b", C.c_double),
                ("vertical", C.c_int), ("n", C.c_double * 2)]


class OrcFillet(C.Structure):
    _fields_ = [("r", C.c_double), ("t1", C.c_double), ("t2", C.c_double), ("p", C.c_double * 2)]


class OrcTool(C.Structure):
    _fields_ = [("num_seg", C.c_int), ("seg", OrcSegment * 5), ("has_fillet", C.c_int), ("fillet", OrcFillet),
                ("mu", C.c_double), ("contact_alpha", C.c_double), ("slave_mass", C.c_double),
                ("vel", C.c_double * 2)]


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            import build_oracle  # noqa: F401  (same directory, on sys.path via conftest/bench)
            build_oracle.build_oracle()
        L = C.CDLL(str(ORACLE_SO))
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_field.restype = C.c_void_p
        L.orc_field.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_constants.argtypes = [C.c_void_p, C.POINTER(OrcPhys), C.POINTER(OrcCorr), C.POINTER(OrcJoco),
                                        C.POINTER(OrcTrml), C.POINTER(OrcTrml)]
        L.orc_set_options.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_set_dt.argtypes = [C.c_void_p, C.c_double]
        L.orc_set_grid_locked.argtypes = [C.c_void_p, C.c_int] + [C.c_double] * 5
        L.orc_set_grid_adaptive.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_get_geometry.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_cells.restype = C.c_void_p
        L.orc_cells.argtypes = [C.c_void_p, C.c_int]
        L.orc_num_cell.argtypes = [C.c_void_p]
        L.orc_set_tool.argtypes = [C.c_void_p, C.POINTER(OrcTool)]
        L.orc_set_reference_functions.argtypes = [C.c_void_p] * 5
        L.orc_get_tool.argtypes = [C.c_void_p, C.POINTER(OrcTool)]
        for f in ("orc_grid_update", "orc_step"):
            getattr(L, f).argtypes = [C.c_void_p]
        for f in ("orc_stage_predict", "orc_stage_interact", "orc_stage_rates", "orc_stage_finish"):
            getattr(L, f).argtypes = [C.c_void_p]
        L.orc_steps.argtypes = [C.c_void_p, C.c_int]
        L.orc_steps_force_log.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_usui.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_void_p]
        L.orc_report_force.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_out_of_grid.restype = C.c_longlong
        L.orc_out_of_grid.argtypes = [C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_cubic_spline.argtypes = [C.c_double] * 5 + [C.c_void_p]
        L.orc_lapl_pse.restype = C.c_double
        L.orc_lapl_pse.argtypes = [C.c_double] * 5
        L.orc_sigma_yield.restype = C.c_double
        L.orc_sigma_yield.argtypes = [C.POINTER(OrcJoco), C.c_double, C.c_double, C.c_double]
        L.orc_sigma_yield_tanh.restype = C.c_double
        L.orc_sigma_yield_tanh.argtypes = [C.POINTER(OrcJoco), C.c_double, C.c_double, C.c_double]
        L.orc_solve_secant.restype = C.c_double
        L.orc_solve_secant.argtypes = [C.POINTER(OrcJoco), C.c_int] + [C.c_double] * 7 + [C.c_void_p]
        L.orc_line_from_points.argtypes = [C.c_double] * 4 + [C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def ref():
    """The reference's host-compiled sources, or None where they were not built."""
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            return None
        L = C.CDLL(str(REF_SO))
        L.refh_cubic_spline.argtypes = [C.c_double] * 5 + [C.c_void_p]
        L.refh_usui.argtypes = [C.c_int] + [C.c_void_p] * 7 + [C.c_double] * 5 + [C.c_void_p]
        L.refh_lapl_pse.restype = C.c_double
        L.refh_lapl_pse.argtypes = [C.c_double] * 5
        L.refh_sigma_yield.restype = C.c_double
        L.refh_sigma_yield.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.refh_sigma_yield_tanh.restype = C.c_double
        L.refh_sigma_yield_tanh.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.refh_solve_secant.restype = C.c_double
        L.refh_solve_secant.argtypes = [C.c_void_p, C.c_int] + [C.c_double] * 7
        L.refh_solve_secant_jc.restype = C.c_double
        L.refh_solve_secant_jc.argtypes = [C.c_void_p] + [C.c_double] * 7
        L.refh_tool_create.argtypes = [C.c_double] * 8
        L.refh_tool_create_points.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.refh_tool_dump.argtypes = [C.c_void_p] * 3
        L.refh_tool_set_vel.argtypes = [C.c_double, C.c_double]
        L.refh_tool_update.argtypes = [C.c_double]
        L.refh_tool_sample.argtypes = [C.c_double, C.c_void_p, C.c_int]
        L.refh_tool_safe_bb.argtypes = [C.c_double, C.c_void_p]
        L.refh_line_from_points.argtypes = [C.c_double] * 4 + [C.c_void_p]
        L.refh_setup_ref_cut.argtypes = [C.c_int] + [C.c_double] * 5
        L.refh_setup_rings.argtypes = [C.c_int]
        L.refh_setup_impact.argtypes = [C.c_int]
        L.refh_get_array.argtypes = [C.c_int, C.c_void_p]
        L.refh_get_constants.argtypes = [C.c_void_p]
        L.refh_get_grid.argtypes = [C.c_void_p]
        L.refh_get_scene_tool.argtypes = [C.c_void_p] * 4
        L.refh_get_grid_max_cell.restype = C.c_int
        _ref = L
    return _ref


REF_GPU_SO = HERE / "_ref" / "libref_gpu.so"
REF_GPU_PSE_SO = HERE / "_ref" / "libref_gpu_pse.so"
_ref_gpu = {}


def ref_gpu(solver: str = "brookshaw"):
    """The reference's own FP64 CUDA step (oracle/_ref/libref_gpu.so; solver="pse": its PSE heat
    solver build, libref_gpu_pse.so), or None where it was not built. Needs a CUDA device to
    run."""
    if solver not in _ref_gpu:
        so = REF_GPU_PSE_SO if solver == "pse" else REF_GPU_SO
        if not so.exists():
            return None
        L = C.CDLL(str(so))
        vp, d, i = C.c_void_p, C.c_double, C.c_int
        L.refg_create.argtypes = [i] + [vp] * 7 + [d] * 5
        L.refg_geometry.argtypes = [vp, vp]
        L.refg_geometry.restype = None
        L.refg_set_constants.argtypes = [vp] * 5 + [d]
        L.refg_set_tool.argtypes = [C.POINTER(OrcTool), vp]
        L.refg_get_tool.argtypes = [C.POINTER(OrcTool)]
        L.refg_set_field.argtypes = [i, vp]
        L.refg_get_field.argtypes = [i, vp]
        L.refg_step.argtypes = [i]
        L.refg_run_timed.argtypes = [i, vp]
        L.refg_get_cells.argtypes = [vp, vp]
        L.refg_report_force.argtypes = [vp]
        _ref_gpu[solver] = L
    return _ref_gpu[solver]


class RefGPU:
    """One system of the reference's own FP64 CUDA build (one per process at a time: the
    reference keeps its constants and options process-wide)."""

    def __init__(self, st: dict, phys7, corr6, joco12, trml_wp6, trml_tool6, tool: OrcTool,
                 solver: str = "brookshaw"):
        self.L = ref_gpu(solver)
        if self.L is None:
            raise RuntimeError(f"reference GPU build missing ({solver})")
        self.N = int(st["N"])
        a = {k: np.ascontiguousarray(st[k], dtype=np.float64) for k in ("pos", "vel", "rho", "T", "h", "fixed",
                                                                         "tool_p")}
        bbmin, bbmax, h = st["grid"]
        rc = self.L.refg_create(self.N, *[_ptr(a[k]) for k in ("pos", "vel", "rho", "T", "h", "fixed", "tool_p")],
                                bbmin[0], bbmin[1], bbmax[0], bbmax[1], h)
        self._check(rc, "refg_create")
        self._c = [np.ascontiguousarray(x, dtype=np.float64) for x in (phys7, corr6, joco12, trml_wp6, trml_tool6)]
        self._tool = tool
        self._check(self.L.refg_set_tool(C.byref(tool), _ptr(self._c[0])), "refg_set_tool")
        self._check(self.L.refg_set_constants(*[_ptr(x) for x in self._c], st["dt"]), "refg_set_constants")

    @staticmethod
    def _check(rc, where):
        if rc != 0:
            raise RuntimeError(f"{where} failed ({rc})")

    def set_field(self, name: str, values) -> None:
        fid, w = FIELDS[name]
        dt = np.int32 if name in INT_FIELDS else np.float64
        v = np.ascontiguousarray(np.asarray(values, dtype=dt).reshape(self.N * w))
        self._check(self.L.refg_set_field(fid, _ptr(v)), "refg_set_field")

    def get(self, name: str) -> np.ndarray:
        fid, w = FIELDS[name]
        dt = np.int32 if name in INT_FIELDS else np.float64
        out = np.zeros(self.N * w, dtype=dt)
        self._check(self.L.refg_get_field(fid, _ptr(out)), "refg_get_field")
        return out.reshape(self.N, w) if w > 1 else out

    def step(self, n: int = 1) -> None:
        self._check(self.L.refg_step(n), "refg_step")

    def run_timed(self, n: int) -> float:
        ms = C.c_float()
        self._check(self.L.refg_run_timed(n, C.byref(ms)), "refg_run_timed")
        return float(ms.value)

    def geometry(self):
        i3 = np.zeros(3, dtype=np.int32)
        d3 = np.zeros(3)
        self.L.refg_geometry(_ptr(i3), _ptr(d3))
        return {"nx": int(i3[0]), "ny": int(i3[1]), "num_cell": int(i3[2]), "bbmin_x": d3[0], "bbmin_y": d3[1],
                "dx": d3[2]}

    def cells(self):
        nc = self.geometry()["num_cell"]
        st = np.zeros(nc, dtype=np.int32)
        en = np.zeros(nc, dtype=np.int32)
        self._check(self.L.refg_get_cells(_ptr(st), _ptr(en)), "refg_get_cells")
        return st, en

    def report_force(self):
        out = np.zeros(2)
        self._check(self.L.refg_report_force(_ptr(out)), "refg_report_force")
        return out

    def get_tool(self) -> OrcTool:
        t = OrcTool()
        self._check(self.L.refg_get_tool(C.byref(t)), "refg_get_tool")
        return t


def use_reference_functions(o) -> bool:
    """Run oracle state `o` on the reference's own host-compiled per-particle functions
    (kernels.cuh cubic_spline, lapl_pse; plasticity.cuh sigma_yield, solve_secant) instead of
    the restatements; False (nothing changed) where the reference's sources were not built."""
    R = ref()
    if R is None:
        return False
    fns = [C.cast(getattr(R, n), C.c_void_p) for n in
           ("refh_cubic_spline", "refh_lapl_pse", "refh_sigma_yield", "refh_solve_secant_jc")]
    o.L.orc_set_reference_functions(o.s, *fns)
    o._ref_fns = fns
    return True


def joco_struct(jc12) -> OrcJoco:
    return OrcJoco(*[float(v) for v in jc12])


class Oracle:
    """Owns one oracle state (particle_gpu + grid + leap_frog + constants + tool)."""

    def __init__(self, N: int):
        self.L = lib()
        self.N = int(N)
        self.s = self.L.orc_create(self.N)

    def __del__(self):
        try:
            if self.s:
                self.L.orc_destroy(self.s)
                self.s = None
        except Exception:
            pass

    def field(self, name: str) -> np.ndarray:
        """A live numpy view of a field (re-fetch after every sort: the Green grid swaps)."""
        fid, w = FIELDS[name]
        p = self.L.orc_field(self.s, fid)
        dt = C.c_int if name in INT_FIELDS else C.c_double
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(dt)), shape=(self.N * w,))
        return arr.reshape(self.N, w) if w > 1 else arr

    def set_field(self, name: str, values) -> None:
        v = self.field(name)
        v[...] = np.asarray(values, dtype=v.dtype).reshape(v.shape)

    def get(self, name: str) -> np.ndarray:
        return self.field(name).copy()

    def cells(self):
        nc = self.L.orc_num_cell(self.s)
        st = np.ctypeslib.as_array(C.cast(self.L.orc_cells(self.s, 0), C.POINTER(C.c_int)), shape=(nc,)).copy()
        en = np.ctypeslib.as_array(C.cast(self.L.orc_cells(self.s, 1), C.POINTER(C.c_int)), shape=(nc,)).copy()
        return st, en

    def geometry(self):
        i3 = np.zeros(3, dtype=np.int32)
        d5 = np.zeros(5)
        self.L.orc_get_geometry(self.s, _ptr(i3), _ptr(d5))
        return {"nx": int(i3[0]), "ny": int(i3[1]), "num_cell": int(i3[2]), "bbmin_x": d5[0],
                "bbmin_y": d5[1], "bbmax_x": d5[2], "bbmax_y": d5[3], "dx": d5[4]}

    def report_force(self):
        out = np.zeros(2)
        self.L.orc_report_force(self.s, _ptr(out))
        return out

    def usui(self, K, alpha, tool_vel):
        out = np.zeros(3)
        self.L.orc_usui(self.s, K, alpha, tool_vel[0], tool_vel[1], _ptr(out))
        return out

    def steps_force_log(self, n: int):
        """n steps; the (Fc, Ff) of report_force after each one, shape (n, 2)."""
        out = np.zeros((n, 2))
        if self.L.orc_steps_force_log(self.s, n, _ptr(out)) != 0:
            raise RuntimeError("oracle step failed")
        return out

    def get_tool(self) -> OrcTool:
        t = OrcTool()
        self.L.orc_get_tool(self.s, C.byref(t))
        return t
