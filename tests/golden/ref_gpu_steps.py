"""Golden vectors of the reference's own FP64 CUDA step (test infrastructure).

The reference's device sources, compiled unchanged for sm_100a (oracle/_ref/libref_gpu.so, its
Brookshaw heat solver, and libref_gpu_pse.so, its PSE solver), step a small compressive scene
(setup_ref_cut at ny = 6, perturbed with seed 51; 592 particles, the tool in contact) twice
through leap_frog::step on a GPU. The state and rates after the second step are kept here, so that
the CPU suite checks the oracle's whole step bodies (pair loop, actions, contact, sort, and the PSE
sums) against outputs the reference itself produced, on machines without a GPU. The scene is
compressive so that the artificial stress stays zero on both sides for these steps (where it is
nonzero the oracle's glibc float trigonometry and CUDA's differ by a few float ulps).

Written on a machine with a CUDA device and the reference builds by
`python tests/golden/make_golden.py ref_gpu`; checked by tests/test_oracle_ref_gpu_golden.py.
"""
from __future__ import annotations

import ctypes as C
import hashlib

import numpy as np

NY, SEED, STEPS = 6, 51, 2
SOLVERS = {"brookshaw": 0, "pse": 1}  # the oracle's thermal solver numbers (MF_THERMAL_*)
FIELDS = ("pos", "vel", "S", "rho", "T", "fc", "ft", "pos_t", "vel_t", "S_t", "rho_t", "T_t")
INDEX_FIELDS = ("idx", "hash", "blanked")
INPUT_FIELDS = ("pos", "vel", "rho", "T", "S", "fc", "ft", "n")


def state(mf):
    """The fixture's input state, regenerated from the product's host scene code (bit for bit the
    reference's setup_ref_cut) and numpy's seeded generator."""
    from helpers import perturbed_scene

    return perturbed_scene(mf, ny=NY, seed=SEED, tensile=False)


def digest(st) -> str:
    h = hashlib.sha256()
    for k in INPUT_FIELDS:
        h.update(np.ascontiguousarray(st[k], dtype=np.float64).tobytes())
    return h.hexdigest()


def _doubles(struct):
    return [getattr(struct, f) for f, _ in struct._fields_]


def compute(mf, orc) -> dict:
    out = {}
    for name in SOLVERS:
        st = state(mf)
        tool = orc.OrcTool()
        C.memmove(C.byref(tool), C.byref(st["tool"]), C.sizeof(orc.OrcTool))
        r = orc.RefGPU(st, _doubles(st["phys"]), _doubles(st["corr"]), _doubles(st["joco"]),
                       _doubles(st["trml_wp"]), _doubles(st["trml_tool"]), tool, solver=name)
        for k in ("S", "eps_pl", "eps_pl_dot", "fc", "ft", "n", "pos_t", "vel_t", "rho_t", "S_t", "T_t", "blanked"):
            r.set_field(k, st[k])
        r.step(STEPS)
        wp = r.get("tool_p") == 0.0
        assert np.all(r.get("R")[wp] == 0.0), "the artificial stress became nonzero"
        assert np.count_nonzero(np.abs(r.get("fc")).sum(axis=1)) > 5, "no particle in contact"
        for k in FIELDS + INDEX_FIELDS:
            out[f"{name}_{k}"] = r.get(k)
        out[f"{name}_force"] = r.report_force()
        out[f"{name}_N"] = np.array(st["N"])
        out[f"{name}_input_digest"] = np.array(digest(st))
    return out
