"""Build recipe for the in-tree CUDA library ``openaccel_b200/_lib/libopenaccel_b200.so``.

The kernels are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``)
with nvcc; the shared library exports the C-ABI declared in
``include/openaccel_b200.h``. Run ``python -m openaccel_b200.build``.
"""
from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libopenaccel_b200.so")
SOURCES = ["oa_kernels.cu", "oa_krylov.cu", "oa_amg.cu", "oa_capi.cu", "oa_static_solve.cu", "oa_scalar_solve.cu",
           "oa_diffusion.cu", "oa_sst.cu"]
HEADERS = ["oa_geom.cuh", "oa_hex8.cuh", "oa_tet4.cuh", "oa_rowlane.cuh", "oa_internal.h", "oa_krylov.h", "oa_amg.h",
           "oa_amg_symbolic.h", "oa_tet4_lists.h", "oa_hex_orient.h",
           "oa_scalar_solve.h", "oa_graph.h"]

NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-O3",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "openaccel_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every CUDA source for sm_100a and link the shared library."""
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = [os.path.join(LIBDIR, src.replace(".cu", ".o")) for src in SOURCES]

    def compile_one(src, obj):
        cmd = [NVCC, *FLAGS, "-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        for f in [ex.submit(compile_one, s, o) for s, o in zip(SOURCES, objs)]:
            f.result()
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp, "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
