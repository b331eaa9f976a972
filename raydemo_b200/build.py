"""Builds libraygpu.so (sm_100a) in-tree with nvcc.

Every translation unit is compiled with --fmad=false and the host compiler
with -ffp-contract=off: the closest-hit, triangle-precompute and ray-hash
arithmetic must round every product and sum on its own, as the reference
build does.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libraygpu.so")
OBJ_DIR = os.path.join(OUT_DIR, "obj")

SOURCES = ["api.cu", "bvh_build.cu", "radix_sort.cu", "trace.cu", "sort.cu", "sort_noalloc.cu", "render.cu", "render_kernels.cu",
           "scene_shading.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
                     "-Xptxas", "-warn-spills", "-DNDEBUG"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _needs(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra_flags: list[str] | None = None) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "raygpu.h"))
    cmds = []
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _needs(o, [s] + headers + [__file__]):
            cmds.append([nvcc()] + NVCC_FLAGS + (extra_flags or []) + ["-c", s, "-o", o])

    def run(cmd):
        p = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, p

    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for cmd, p in ex.map(run, cmds):
            if verbose or p.returncode != 0:
                sys.stdout.write(" ".join(cmd) + "\n" + p.stdout + p.stderr)
            if p.returncode != 0:
                raise RuntimeError(f"nvcc failed on {cmd[-3]}")
    if force or cmds or not os.path.exists(LIB):
        link = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-lpthread"]
        p = subprocess.run(link, capture_output=True, text=True)
        if verbose or p.returncode != 0:
            sys.stdout.write(" ".join(link) + "\n" + p.stdout + p.stderr)
        if p.returncode != 0:
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
