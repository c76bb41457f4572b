"""Build libaak_b200.so in-tree for sm_100a (B200).

    python -m emri_kludge_suite_b200.build [--force] [--verbose]

Each translation unit is compiled with nvcc into ``_build/`` (skipped when the
object is newer than its sources and headers) and linked into
``emri_kludge_suite_b200/libaak_b200.so``.  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libaak_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", os.path.join(REPO, "include")]

# per-file flags: the device map solve and the device AK evolution round as the host does (no FMA contraction)
FILE_FLAGS = {"kernels/parmap_newton.cu": ["-fmad=false"], "kernels/ak_evolve.cu": ["-fmad=false"]}

SOURCES = [
    "host/kerr.cpp",
    "host/inspiral.cpp",
    "host/pipeline.cpp",
    "host/parmap_data.cpp",
    "host/shard.cpp",
    "kernels/aak_dense.cu",
    "kernels/likelihood.cu",
    "kernels/parmap_mlp.cu",
    "kernels/parmap_newton.cu",
    "kernels/ak_evolve.cu",
    "capi/aak_capi.cpp",
    "capi/mlp_capi.cpp",
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libaak_b200.so")


def _headers():
    found = []
    for pat in ("*.h", "*.hpp", "*.cuh"):
        found += glob.glob(os.path.join(CSRC, "**", pat), recursive=True)
    return found + glob.glob(os.path.join(REPO, "include", "*.h"))


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    hdrs = _headers()
    extra = list(extra_flags or []) + os.environ.get("AAK_EXTRA_NVCC_FLAGS", "").split()
    jobs = []
    objs = []
    for rel in SOURCES:
        src = os.path.join(CSRC, rel)
        obj = os.path.join(BUILD, rel.replace("/", "_") + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            cmd = [cc, *ARCH, *COMMON, *FILE_FLAGS.get(rel, []), *extra, "-c", src, "-o", obj]
            if rel.endswith(".cu"):
                cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, flush=True)

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(run, jobs))
    if force or jobs or not os.path.exists(LIB) or _stale(LIB, objs):
        cmd = [cc, *ARCH, "-shared", "-o", LIB, *objs, "-lcufft", "-lcudart", "-lpthread"]
        run(cmd)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
