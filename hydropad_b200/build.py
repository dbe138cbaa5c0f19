"""Build recipe of the CUDA library (libhydropad_b200.so, in-tree).

Every kernel is compiled for sm_100a only, without implicit multiply-add
contraction (--fmad=false): the FP64 kernels then round like the reference's
scalar Fortran, and every kernel gives the same bits in every tile shape and
in batched launches.  The mixed-precision kernels also use the hardware
approximations of FP32 division and square root (-use_fast_math); fused
multiply-adds there are written explicitly.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD_DIR = os.path.join(ROOT, "_build")
LIB_NAME = "libhydropad_b200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]
MIXED = ["-use_fast_math", "--fmad=false"]
SOURCES = [
    ("hp_kernels_fp64.cu", ["--fmad=false"]),
    # FP32 stages may use the hardware approximations (FP64 is unaffected).
    # No implicit contraction either: ptxas may contract a multiply-add
    # differently in different instantiations (tiles, batched or not), and
    # a box must give the same bits whatever tile or batch it runs in.
    ("hp_kernels_mixed.cu", MIXED),
    # sweeps with the static gravity source, same flags as above
    ("hp_kernels_grav_fp64.cu", ["--fmad=false"]),
    ("hp_kernels_grav_mixed.cu", MIXED),
    # the non-STENCIL build's full-pencil solver (FP64), same flags
    ("hp_kernels_pencil_fp64.cu", ["--fmad=false"]),
    # persistent batched sweeps (many boxes per launch), same flags as above
    ("hp_batch_fp64.cu", ["--fmad=false"]),
    ("hp_batch_mixed.cu", MIXED),
    ("hp_api.cu", []),
    ("hp_batch.cu", []),
    ("hp_noalloc.cu", []),
]
HEADERS = ["hp_physics.cuh", "hp_riemann.cuh", "hp_device.cuh", "hp_sweep.cuh", "hp_sweep_ws.cuh", "hp_tma.cuh",
           "hp_sweep_launch.cuh", "hp_launch.h", "hp_ctx.h"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build hydropad_b200")


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile stale objects and link the shared library; return its path."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "hydropad_b200.h")]
    newest_dep = max(_mtime(d) for d in deps)
    objs = []
    cmds = []
    relink = force or not os.path.exists(LIB_PATH)
    for src, extra in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD_DIR, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _mtime(o) < max(_mtime(s), newest_dep):
            cmd = [nvcc, *ARCH, *COMMON, *extra, "-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), file=sys.stderr)
            cmds.append(cmd)
    # translation units compile independently: one nvcc per unit
    if cmds:
        with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
            for r in list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds)):
                sys.stderr.write(r.stderr)
                if r.returncode != 0:
                    raise subprocess.CalledProcessError(r.returncode, r.args, r.stdout, r.stderr)
        relink = True
    if relink or _mtime(LIB_PATH) < max(_mtime(o) for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB_PATH, *objs]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
