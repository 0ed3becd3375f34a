"""Build libsdpx_b200.so (sm_100a) in place with nvcc.

Usage:  python sdpx.jl_b200/build.py [--force]
The library lands next to this file (sdpx.jl_b200/libsdpx_b200.so) so it
travels with the source tree; objects go to sdpx.jl_b200/_build/.
"""
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libsdpx_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]
SOURCES = ["api.cu", "blas_f64.cu", "chol.cu", "vec_kernels.cu", "mixed_f32.cu", "schur_bf16.cu",
           "normal.cu", "certificate.cu", "ozaki.cu", "equality.cu", "sparse_schur.cu",
           "dd_kernels.cu", "batch.cu"]
# Per-file flags.  normal.cu evaluates the reference's scalar cone recurrences
# and must round every product and sum separately (no FMA contraction).
FILE_FLAGS = {"normal.cu": ["--fmad=false"]}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.exists(cand) or cand == "nvcc"):
            return cand
    raise RuntimeError("nvcc not found")


def build(force: bool = False, verbose: bool = False) -> Path:
    from concurrent.futures import ThreadPoolExecutor
    BUILD.mkdir(exist_ok=True)
    deps = sorted(CSRC.glob("*")) + sorted((HERE.parent / "include").glob("*.h")) + [Path(__file__)]
    newest_dep = max(p.stat().st_mtime for p in deps)
    objs, cmds = [], []
    for src in SOURCES:
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < newest_dep:
            cmds.append([nvcc(), *ARCH, *FLAGS, *FILE_FLAGS.get(src, []), "-c", str(CSRC / src),
                         "-o", str(obj)])

    def compile_one(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    # one nvcc per translation unit, in parallel (the objects are independent)
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(compile_one, cmds))
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
