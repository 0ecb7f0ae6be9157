"""Build recipe for the oracle (test infrastructure; never part of the product path).

Three artefacts:

* ``oracle/_build/liboracle.so``: the CPU restatement of the reference step
  (``oracle/sph_oracle.c``), plain C11 + OpenMP, built with gcc.
* ``oracle/_ref/libref_host.so``: the reference's own host-compilable sources, compiled
  where they lie (``<reference>/src``) against the project's GLM-subset shim
  (``oracle/ref_shim``), plus the recording harness ``oracle/ref_host_harness.cu`` and the
  host build of ``plasticity.cuh`` (``oracle/ref_host_plasticity.cpp``). It is only built
  when the reference tree is present; the GPU machines use the prebuilt file or skip.

* ``oracle/_ref/libref_gpu.so``: the reference's own FP64 CUDA step (its device sources,
  unchanged, with the texture shim ``oracle/ref_gpu/ref_texture_shim.h`` force-included) and
  the entry-point harness ``oracle/ref_gpu/ref_gpu_harness.cu``; built where the reference
  tree is present, used on the GPU machine as the GPU oracle and the reference GPU baseline.

All are loaded with ctypes by ``tests/`` and by ``bench.py``'s baseline legs only.
"""
from __future__ import annotations

import os
import shutil
from concurrent.futures import ThreadPoolExecutor
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
# the reference's src/ directory: MF_REFERENCE_SRC, else a reference checkout beside this
# repository (../reference/src); where neither exists only prebuilt files are used
REF_SRC = Path(os.environ.get("MF_REFERENCE_SRC", str(HERE.parent.parent / "reference" / "src")))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CUDA_HOME = Path(NVCC).resolve().parent.parent

ORACLE_LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref_host.so"
REF_GPU_LIB = HERE / "_ref" / "libref_gpu.so"


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(str(c) for c in cmd) + "\n" + r.stdout + "\n")
        raise RuntimeError(f"build step failed: {cmd[0]} ({r.returncode})")
    return r.stdout


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in sources)


def build_oracle(force: bool = False) -> Path:
    """gcc -O2 -fopenmp the C restatement into a shared library (no FMA contraction)."""
    srcs = [HERE / "sph_oracle.c", HERE / "sph_oracle.h"]
    if force or _stale(ORACLE_LIB, srcs):
        ORACLE_LIB.parent.mkdir(parents=True, exist_ok=True)
        _run([
            "gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
            "-fno-fast-math", "-Wall", "-Wno-unused-function",
            "-o", str(ORACLE_LIB), str(HERE / "sph_oracle.c"), "-lm",
        ])
    return ORACLE_LIB


def build_ref(force: bool = False) -> Path | None:
    """Compile the reference's host-side sources (where they lie) into oracle/_ref."""
    if not REF_SRC.is_dir():
        return REF_LIB if REF_LIB.exists() else None
    ref_files = ["benchmarks.cpp", "tool.cpp", "geometric_primitives.cpp", "constants_structs.cpp",
                 "grid.cu"]
    # tool_wear.cu and vtk_writer.cpp are compiled inside ref_host_wear.cu and ref_host_vtk.cu
    # (their device-to-host copies made host copies)
    harness = ["ref_host_harness.cu", "ref_host_wear.cu", "ref_host_vtk.cu"]
    srcs = [HERE / f for f in harness] + [HERE / "ref_host_plasticity.cpp", HERE / "ref_shim" / "glm" / "glm.hpp",
                                          REF_SRC / "tool_wear.cu", REF_SRC / "vtk_writer.cpp"] + \
        [REF_SRC / f for f in ref_files]
    if not (force or _stale(REF_LIB, srcs)):
        return REF_LIB
    obj = HERE / "_ref" / "obj"
    obj.mkdir(parents=True, exist_ok=True)
    inc = ["-I", str(HERE / "ref_shim"), "-I", str(REF_SRC)]
    # the reference's Release flags were -O3 -std=c++11; host code keeps x87-free SSE2
    # arithmetic and no FMA contraction, as gcc does by default for x86-64.
    nv = [NVCC, "-O3", "-std=c++14", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-gencode", "arch=compute_100a,code=sm_100a", "-w", "-x", "cu", "-c"]
    objs = []
    for f in harness:
        o = obj / (Path(f).stem + ".o")
        _run(nv + inc + ["-o", str(o), str(HERE / f)])
        objs.append(o)
    for f in ref_files:
        o = obj / ("ref_" + Path(f).stem + ".o")
        _run(nv + inc + ["-o", str(o), str(REF_SRC / f)])
        objs.append(o)
    o = obj / "ref_host_plasticity.o"
    _run(["g++", "-O3", "-std=c++14", "-fPIC", "-ffp-contract=off", "-w", "-c",
          "-I", str(CUDA_HOME / "include")] + inc + ["-o", str(o), str(HERE / "ref_host_plasticity.cpp")])
    objs.append(o)
    _run([NVCC, "-shared", "-Xcompiler", "-fPIC", "-o", str(REF_LIB)] + [str(x) for x in objs])
    return REF_LIB


def _pse_types_header(out_dir: Path) -> Path:
    """The reference's types.h with its heat-solver switch turned to PSE (types.h selects the
    solver with a #define and no way to override it from the command line): generated from the
    reference's own file at build time into oracle/_ref, never committed, and force-included
    after the texture shim, so that its include guard makes the sources' own types.h a no-op."""
    text = (REF_SRC / "types.h").read_text()
    on, off = "#define Thermal_Conduction_Brookshaw", "//#define Thermal_Conduction_PSE"
    if text.count(on) != 1 or text.count(off) != 1:
        raise RuntimeError("types.h: the heat-solver switch is not where the PSE build expects it")
    text = text.replace(off, "#define Thermal_Conduction_PSE").replace(on, "//#define Thermal_Conduction_Brookshaw")
    out = out_dir / "types_pse.h"
    if not out.exists() or out.read_text() != text:
        out.write_text(text)
    return out


REF_GPU_PSE_LIB = HERE / "_ref" / "libref_gpu_pse.so"


def build_ref_gpu(force: bool = False, solver: str = "brookshaw") -> Path | None:
    """The reference's own FP64 CUDA step for sm_100a (oracle/_ref/libref_gpu.so): its device
    sources compiled unchanged where they lie, with the texture shim force-included and the
    project's GLM subset, plus the entry-point harness oracle/ref_gpu/ref_gpu_harness.cu.
    The reference's own makefile flags: -O3, whole-program per file (no relocatable device
    code); its types.h selects FP64 and the Brookshaw heat solver. solver="pse": the same
    sources built with the switch in types.h turned to its PSE solver
    (oracle/_ref/libref_gpu_pse.so)."""
    pse = solver == "pse"
    lib = REF_GPU_PSE_LIB if pse else REF_GPU_LIB
    if not REF_SRC.is_dir():
        return lib if lib.exists() else None
    ref_files = ["actions_gpu.cu", "interactions_gpu.cu", "leap_frog.cu", "tool_gpu.cu", "grid.cu",
                 "grid_gpu_green.cu", "particle_gpu.cu", "output.cu", "tool.cpp", "geometric_primitives.cpp",
                 "constants_structs.cpp", "types.cpp"]
    shim = HERE / "ref_gpu" / "ref_texture_shim.h"
    harness = HERE / "ref_gpu" / "ref_gpu_harness.cu"
    srcs = [shim, harness, HERE / "ref_shim" / "glm" / "glm.hpp", HERE / "sph_oracle.h", Path(__file__)] + \
        [REF_SRC / f for f in ref_files] + sorted(REF_SRC.glob("*.h")) + sorted(REF_SRC.glob("*.cuh"))
    if not (force or _stale(lib, srcs)):
        return lib
    obj = HERE / "_ref" / ("gpu_obj_pse" if pse else "gpu_obj")
    obj.mkdir(parents=True, exist_ok=True)
    nv = [NVCC, "-O3", "-std=c++14", "-Xcompiler", "-fPIC", "-gencode", "arch=compute_100a,code=sm_100a",
          "-include", str(shim)]
    if pse:
        nv += ["-include", str(_pse_types_header(obj))]
    nv += ["-I", str(HERE / "ref_shim"), "-I", str(REF_SRC), "-I", str(HERE), "-w", "-x", "cu", "-c"]
    jobs = [(obj / ("refg_" + Path(f).stem + ".o"), REF_SRC / f) for f in ref_files]
    jobs.append((obj / "ref_gpu_harness.o", harness))
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        list(pool.map(lambda j: _run(nv + ["-o", str(j[0]), str(j[1])]), jobs))
    objs = [j[0] for j in jobs]
    _run([NVCC, "-shared", "-Xcompiler", "-fPIC", "--cudart", "shared", "-Xlinker", "-Bsymbolic",
          "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(lib)] + [str(x) for x in objs])
    return lib


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
    print(build_ref_gpu(force="--force" in sys.argv))
    print(build_ref_gpu(force="--force" in sys.argv, solver="pse"))
