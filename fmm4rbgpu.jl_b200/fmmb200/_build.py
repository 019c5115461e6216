"""Builds libfmmb200.so (sm_100a) in-tree with nvcc.

Objects go to ``fmm4rbgpu.jl_b200/_build/`` and the library to
``fmm4rbgpu.jl_b200/lib/libfmmb200.so``; both are git-ignored but travel with
the source tree.  Every translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo``.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))  # fmm4rbgpu.jl_b200/
CSRC = os.path.join(PKG_ROOT, "csrc")
OBJ_DIR = os.path.join(PKG_ROOT, "_build")
LIB_DIR = os.path.join(PKG_ROOT, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libfmmb200.so")
INCLUDE = os.path.join(os.path.dirname(PKG_ROOT), "include")

SOURCES = ["sort.cu", "tree.cu", "traverse.cu", "interp.cu", "m2l.cu", "p2p.cu", "backward.cu", "direct.cu", "api.cu",
           "shard.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-diag-suppress", "177"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: cannot build libfmmb200.so")


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    hs.append(os.path.join(INCLUDE, "fmmb200.h"))
    return hs


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def needs_build() -> bool:
    objs = [os.path.join(OBJ_DIR, s.replace(".cu", ".o")) for s in SOURCES]
    srcs = [os.path.join(CSRC, s) for s in SOURCES] + _headers()
    return _stale(LIB_PATH, srcs + objs) or any(_stale(o, srcs) for o in objs)


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    """Compile every .cu for sm_100a and link the shared library; returns its path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()

    def compile_one(src: str):
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
        if not force and not _stale(o, [s] + headers):
            return o
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-I", INCLUDE, "-c", s, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr)
        return o

    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    if force or _stale(LIB_PATH, objs):
        tmp = LIB_PATH + ".tmp"
        cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose=True))
