"""Build the engine's shared library in-tree with nvcc (sm_100a only).

``python -m beamz_b200.build`` compiles ``beamz_b200/csrc/*.cu`` into
``beamz_b200/_fdtd_b200.so``.  The CUDA runtime is linked statically so the
library depends only on the driver; it shares the device's primary context
with PyTorch, so torch-allocated pointers and torch streams are valid in it.

``-fmad=false`` keeps every product and sum separately rounded, in source
order, which is the rounding contract the kernels rely on for parity with
beamz's float32 path; explicit ``fmaf`` calls (the opt-in tolerance arithmetic
of the class step) still emit FFMA.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "_fdtd_b200.so")
SOURCES = ("phase.cu", "fused.cu", "fused3d.cu", "fused_tma.cu", "class_step.cu", "io.cu", "adjoint.cu", "diag.cu", "planner.cu", "analysis.cu", "recorder.cu", "program.cu")
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build beamz_b200")


def flags(extra=()):
    return [
        ARCH, "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", *extra,
    ]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "fdtd_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    """Compile the library if any source is newer than it; return its path."""
    if not force and not needs_build():
        return LIB
    nvcc = nvcc_path()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc, *flags(extra), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = []
    for src, proc in procs:
        out, _ = proc.communicate()
        if verbose and out:
            print(out)
        if proc.returncode != 0:
            failed.append((src, out))
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(f"{s}:\n{o}" for s, o in failed))
    tmp = LIB + ".tmp"
    cmd = [nvcc, ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    res = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if res.returncode != 0:
        raise RuntimeError("link failed:\n" + res.stdout)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    verbose = "-v" in sys.argv
    extra = ("-Xptxas", "-v") if "--ptxas" in sys.argv else ()
    print(build(force=True, verbose=verbose, extra=extra))
