"""Builds fmm_b200/libfmm_b200.so in-tree with nvcc for sm_100a (cross-compiles without a GPU).

    python -m fmm_b200.build [--force] [-v]      # or fmm_b200.build.build()

Every source compiles to its own object in fmm_b200/_build/, the evaluator once per
expansion order (evaluator_order.cu with -DFMMB_P=p), in parallel over the host's cores;
the objects are then linked into the shared library.
"""
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libfmm_b200.so")

SOURCES = ["evaluator.cu", "direct.cu", "tree.cpp", "tables.cpp", "forest.cpp", "helmholtz_tables.cpp",
           "table_cache.cpp", "plan_upload.cpp", "plan_gpu.cu", "p2p_launch.cu"]
ORDER_SOURCE = "evaluator_order.cu"
HEADERS = ["plan.hpp", "evaluator_base.hpp", "evaluator_impl.cuh", "kernels.cuh", "harmonics.cuh", "m2l_tc.cuh",
           "m2l_fused.cuh", "p2p_x2.cuh", "helmholtz.cuh", "helmholtz_far.cuh", "helmholtz_st.cuh", "leaf_far_x2.cuh", "morton.hpp"]

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


def orders():
    """The expansion orders compiled in (FMMB_FOR_EACH_ORDER of evaluator_base.hpp)."""
    text = open(os.path.join(CSRC, "evaluator_base.hpp")).read()
    m = re.search(r"#define FMMB_FOR_EACH_ORDER\(X\)(.*)", text)
    return [int(v) for v in re.findall(r"X\((\d+)\)", m.group(1))]


def _units():
    units = [(os.path.join(CSRC, s), os.path.join(OBJ, os.path.splitext(s)[0] + ".o"), []) for s in SOURCES]
    for p in orders():
        units.append((os.path.join(CSRC, ORDER_SOURCE), os.path.join(OBJ, f"evaluator_p{p}.o"), [f"-DFMMB_P={p}"]))
    return units


def _newest_dependency():
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS + [ORDER_SOURCE]]
    deps.append(os.path.join(ROOT, "include", "fmm_b200.h"))
    deps.append(os.path.abspath(__file__))
    return max(os.path.getmtime(d) for d in deps if os.path.exists(d))


def _stale(path, newest):
    return not os.path.exists(path) or os.path.getmtime(path) < newest


def build(force=False, verbose=False, jobs=None):
    newest = _newest_dependency()
    units = _units()
    if not force and not _stale(OUT, newest) and all(not _stale(o, newest) for _, o, _ in units):
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    todo = [u for u in units if force or _stale(u[1], newest)]

    def compile_one(unit):
        src, obj, extra = unit
        cmd = [NVCC] + FLAGS + extra + (["-Xptxas=-v"] if verbose else []) + ["-c", "-o", obj, src]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return unit, r

    failed = []
    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as pool:
        for (src, obj, extra), r in pool.map(compile_one, todo):
            if verbose or r.returncode:
                sys.stderr.write(f"== {os.path.basename(obj)}\n{r.stdout}{r.stderr}")
            if r.returncode:
                failed.append(os.path.basename(obj))
    if failed:
        raise RuntimeError("nvcc failed for " + ", ".join(failed))
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT] + [o for _, o, _ in units]
    subprocess.run(link, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
