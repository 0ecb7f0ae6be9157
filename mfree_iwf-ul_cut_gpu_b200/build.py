"""Build the product library ``lib/libmfree_b200.so`` (sm_100a, in-tree).

    python mfree_iwf-ul_cut_gpu_b200/build.py [--force] [--ptxas-verbose]

nvcc compiles the CUDA translation unit for ``arch=compute_100a,code=sm_100a`` with
``-lineinfo``; the host scene/tool code is plain C++17. The library is built in the source
tree so that it travels with the repository to the GPU machine.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libmfree_b200.so"
# benchmark-only measurement aid (FP64 FMA peak, pow/log/division latency), kept out of the
# product library
PROBE_SRC = PKG / "probe" / "mf_probe.cu"
PROBE_LIB = LIB_DIR / "libmf_probe.so"
OBJ = PKG / "_build"
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-I", str(ROOT / "include"), "-I", str(CSRC)] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-I", str(ROOT / "include")]


def _run(cmd):
    r = subprocess.run([str(c) for c in cmd], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(str(c) for c in cmd) + "\n" + r.stdout + "\n")
        raise RuntimeError(f"build failed: {cmd[0]}")
    return r.stdout


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _stale(target: Path) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    deps = list(CSRC.glob("*")) + list((ROOT / "include").glob("*.h")) + [Path(__file__)]
    return any(d.stat().st_mtime > t for d in deps)


def build_probe(force: bool = False) -> Path:
    """The benchmark's FP64 probe library (lib/libmf_probe.so)."""
    if force or not PROBE_LIB.exists() or PROBE_SRC.stat().st_mtime > PROBE_LIB.stat().st_mtime:
        LIB_DIR.mkdir(parents=True, exist_ok=True)
        _run([NVCC] + NVCC_FLAGS + ["-shared", "-o", PROBE_LIB, PROBE_SRC, "-lcudart"])
    return PROBE_LIB


def build(force: bool = False, ptxas_verbose: bool = False) -> Path:
    build_probe(force)
    if not force and not _stale(LIB):
        return LIB
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    objs = []
    cmds = []
    for src in sources():
        o = OBJ / (src.stem + ".o")
        if src.suffix == ".cu":
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            cmds.append([NVCC] + NVCC_FLAGS + extra + ["-c", "-o", o, src])
        else:
            cmds.append(["g++"] + CXX_FLAGS + ["-c", "-o", o, src])
        objs.append(o)
    # the translation units compile independently: side by side
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        log = list(pool.map(_run, cmds))
    tmp = LIB.with_suffix(".so.tmp")
    _run([NVCC, "-shared", "-Xcompiler", "-fPIC"] + ARCH + ["-o", tmp] + objs + ["-lcudart"])
    tmp.replace(LIB)
    if ptxas_verbose:
        print("\n".join(x for x in log if x.strip()))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, ptxas_verbose="--ptxas-verbose" in sys.argv))
