"""Builds libisg.so in-tree for sm_100a (explicit nvcc, no JIT cache).

    python inverse-solver-gpu_b200/build.py [--force] [-j N]

Objects go to inverse-solver-gpu_b200/_build/, the library to
inverse-solver-gpu_b200/isg/libisg.so.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "isg", "libisg.so")
REFAPI_SRC = os.path.join(HERE, "refapi", "isg_refapi.cpp")
REFAPI_OUT = os.path.join(HERE, "isg", "libisg_ref.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
           "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def deps(src: str) -> list[str]:
    return [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))] + \
        [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]


def stale(target: str, inputs: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in inputs if os.path.exists(p))


def compile_one(src: str, force: bool, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if force or stale(obj, deps(src)):
        lang = [] if src.endswith(".cu") else ["-x", "cu"]
        cmd = [nvcc(), *ARCH, *NVFLAGS, *extra, *lang, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if r.stderr.strip():
            sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, jobs: int = 8, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, extra), sources()))
    if force or stale(OUT, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_refapi(force)
    return OUT


def build_refapi(force: bool = False) -> str:
    """libisg_ref.so: the reference's routine names over libisg.so.  Its globals
    (res, level, ...) stay undefined until the caller's driver links it."""
    inputs = [REFAPI_SRC, OUT, os.path.join(ROOT, "include", "isg_refapi.h"), os.path.join(ROOT, "include", "isg.h")]
    if force or stale(REFAPI_OUT, inputs):
        cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc())), "include")
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I" + cuda_inc, "-o", REFAPI_OUT, REFAPI_SRC,
               "-L" + os.path.dirname(OUT), "-lisg", "-L" + os.path.join(os.path.dirname(cuda_inc), "lib64"),
               "-lcudart", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"libisg_ref.so failed:\n{r.stdout}\n{r.stderr}")
    return REFAPI_OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.ptxas_v))
