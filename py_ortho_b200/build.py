"""Builds libmvs_b200.so (sm_100a) in-tree with nvcc.

Usage: ``python -m py_ortho_b200.build [--force] [--verbose]``. Objects go to
``py_ortho_b200/_build/``; the shared library to ``py_ortho_b200/libmvs_b200.so``.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmvs_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-I", INCLUDE]
# per-file extra flags: PatchMatch and the pass-2 geometry are evaluated without contraction
# (one rounding per written operation, as the reference's C evaluates them)
EXTRA = {
    "patchmatch.cu": ["-fmad=false"],
    "views.cu": ["-fmad=false"],
    "height.cu": ["-fmad=false"],
}
SOURCES = ["helpers.cu", "sweep.cu", "patchmatch.cu", "batch.cu", "noalloc.cu", "views.cu", "height.cu"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmvs_b200")
    return p


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False, debug_bounds: bool = False) -> str:
    """Compiles the library; debug_bounds: the bounds-checked build (-DMVS_DEBUG_BOUNDS) into
    libmvs_b200_debug.so, objects under _build/debug."""
    build_dir = os.path.join(BUILD, "debug") if debug_bounds else BUILD
    lib = LIB.replace("libmvs_b200.so", "libmvs_b200_debug.so") if debug_bounds else LIB
    flags = ["-DMVS_DEBUG_BOUNDS"] if debug_bounds else []
    os.makedirs(build_dir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(INCLUDE, "mvs_b200.h"))
    objs = []
    jobs = []
    cc = nvcc()
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(build_dir, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or ptxas_info or _stale(obj, [path] + headers):
            cmd = [cc, "-c", path, "-o", obj] + ARCH + COMMON + EXTRA.get(src, []) + flags
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            jobs.append((src, cmd))
    # the translation units compile in parallel (one nvcc per source file)
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda j: (j[0], subprocess.run(j[1], capture_output=True, text=True)), jobs))
    for src, r in results:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if ptxas_info or verbose:
            sys.stdout.write(r.stdout + r.stderr)
    if force or _stale(lib, objs):
        tmp = lib + ".partial"              # linked aside, then moved into place in one step
        cmd = [cc, "-shared", "-o", tmp] + objs + ARCH + ["-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, lib)
    return lib


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills per kernel")
    ap.add_argument("--debug-bounds", action="store_true",
                    help="the bounds-checked debug build (libmvs_b200_debug.so)")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose, a.ptxas_info, a.debug_bounds))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
