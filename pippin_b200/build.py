"""Build the CUDA backend library (lib/libpippin_b200.so) for sm_100a.

Compiles pippin_b200/csrc with nvcc into a shared library kept inside the
package directory, so it travels with the source tree. Run as a module
(`python -m pippin_b200.build`) or call build().
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpippin_b200.so")
SOURCES = ["pg_kernels.cu", "pg_api.cpp", "pg_peak.cu", "pg_noalloc.cu", "pg_mlp.cu", "pg_render.cu"]
# the rasteriser rounds every product and sum on its own (no FMA contraction),
# so that its coverage, depth and shading match an IEEE single-precision
# evaluation of the same expressions on the CPU bit for bit
EXTRA_FLAGS = {"pg_render.cu": ["-fmad=false"]}
HEADERS = ["pg_math.cuh", "pg_model.h", "pg_tile.cuh", "pg_dynamics.cuh", "pg_collide.cuh", "pg_linalg.cuh", "pg_small.cuh", "pg_pgs.cuh", "pg_general.cuh", "pg_mlp.h",
           "pg_newton.cuh", "pg_kernels.h"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(HERE, "..", "include", h)
             for h in ("pippin_b200.h", "pippin_b200_tools.h", "pippin_b200_mlp.h", "pippin_b200_render.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if a source is newer than it; returns its path."""
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(LIBDIR, src.rsplit(".", 1)[0] + ".o")
        cmd = [_nvcc(), *NVCC_FLAGS, *EXTRA_FLAGS.get(src, []), "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd = [_nvcc(), *NVCC_FLAGS, "-x", "cu", "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp, "-cudart", "static"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
