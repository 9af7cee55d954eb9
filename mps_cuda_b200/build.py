"""Build recipe of the native library ``libmps_b200.so`` (sm_100a).

The library is plain nvcc output: CUDA kernels and the C-ABI of ``include/mps_b200.h`` in one
shared object, built in-tree next to this file so that it travels with the repository.

Flags that matter for results:
  -fmad=false                 no implicit multiply-add contraction; every fused multiply-add
                              in the kernels is an explicit __fma_rn
  -Xcompiler -ffp-contract=off  same rule for host code (derived constants)
  no --use_fast_math          IEEE division and square root
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmps_b200.so")
SOURCES = ["mps_api.cu", "mps_inst_f32.cu", "mps_inst_f64.cu", "mps_inst_mix.cu",
           "mps_noalloc.cu", "mps_scene.cpp", "mps_io.cpp", "mps_output.cu", "mps_peaks.cu"]
HEADERS = ["mps_types.h", "mps_device.cuh", "mps_kernels.cuh", "mps_adjoint.cuh", "mps_solver.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(ROOT, "include", "mps_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(f) <= t for f in _inputs() if os.path.exists(f))


COMMON = ["-lineinfo", "-O3", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
          "-Xcompiler", "-fPIC,-ffp-contract=off,-O2"]


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compile every translation unit (in parallel) and link libmps_b200.so."""
    if not force and up_to_date():
        return LIB
    nvcc = nvcc_path()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc, *ARCH, *COMMON, "-Xptxas", "-warn-spills", "-c", os.path.join(CSRC, src),
               "-o", obj]
        if extra:
            cmd += extra
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, obj, subprocess.Popen(cmd, cwd=CSRC, stdout=subprocess.PIPE,
                                                 stderr=subprocess.STDOUT, text=True)))
    objs, errors = [], []
    for src, obj, pr in procs:
        out, _ = pr.communicate()
        if pr.returncode != 0:
            errors.append(f"{src}:\n{out}")
        elif verbose and out:
            print(out, file=sys.stderr)
        objs.append(obj)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    cmd = [nvcc, *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lpthread"]
    res = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else None
    print(build(force=True, verbose=v or bool(extra), extra=extra))
