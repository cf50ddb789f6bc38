"""Builds fmm_b200/libfmm_b200.so in-tree with nvcc for sm_100a (cross-compiles without a GPU).

    python -m fmm_b200.build          # or fmm_b200.build.build()
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libfmm_b200.so")

SOURCES = ["evaluator.cu", "direct.cu", "tree.cpp", "tables.cpp", "forest.cpp", "helmholtz_tables.cpp"]
HEADERS = ["plan.hpp", "kernels.cuh", "harmonics.cuh", "m2l_tc.cuh", "m2l_fused.cuh", "p2p_x2.cuh", "helmholtz.cuh"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3",
    "--expt-relaxed-constexpr",
    # f32 denormals flush to zero: every r^2 that reaches rsqrt is >= 2^-108 (normal), and
    # the P2P rsqrt is then one MUFU instruction; f64 is unaffected
    "-ftz=true",
    "-ccbin", "g++",
]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "fmm_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not _stale():
        return OUT
    cmd = [NVCC] + FLAGS + ["-shared", "-o", OUT] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
