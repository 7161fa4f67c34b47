"""Builds the CUDA library of the package in-tree for sm_100a.

Outputs (git-ignored, shipped with the source tree):
  213transpose_b200/lib213transpose_b200.so   the C ABI of include/t213.h
  lib/libinplacett.a                          the reference-compatible C++ API
                                              (inplace::transpose<T> & co.)
  213transpose_b200/bin/test_213inplace, gen_ans   the reference's drivers

Usage: python 213transpose_b200/build.py [-j N] [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
SO = os.path.join(PKG, "lib213transpose_b200.so")
LIBDIR = os.path.join(ROOT, "lib")
STATIC = os.path.join(LIBDIR, "libinplacett.a")
BINDIR = os.path.join(PKG, "bin")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC,
                     "--expt-relaxed-constexpr"]

LIB_SOURCES = ["runtime.cu", "launch_gather.cu", "launch_cycles.cu", "launch_tiles.cu", "host_io.cu",
               "tuner.cu", "batch.cu", "serve.cu", "noalloc.cu"]
CXX_API_SOURCES = ["cxx_api.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps_newer(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    for d in [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
            [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]:
        if os.path.getmtime(d) > t:
            return True
    return False


def compile_one(src: str, force: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src).rsplit(".", 1)[0] + ".o")
    if force or _deps_newer(obj, src):
        cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(jobs: int | None = None, force: bool = False, drivers: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    extra = [os.path.join(CSRC, s) for s in CXX_API_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force), srcs + extra))
    lib_objs = objs[:len(srcs)]
    if force or not os.path.exists(SO) or any(os.path.getmtime(o) > os.path.getmtime(SO) for o in lib_objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", SO] + lib_objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if extra:
        os.makedirs(LIBDIR, exist_ok=True)
        if os.path.exists(STATIC):
            os.remove(STATIC)
        subprocess.run(["ar", "rcs", STATIC] + lib_objs + objs[len(srcs):], check=True)
        if drivers:
            build_drivers()
    return SO


def build_drivers() -> None:
    """The reference's two drivers with its argv and output format:
    test_213inplace (the GPU path, linked against lib/libinplacett.a) and
    gen_ans (the host answer generator, plain C++ with no GPU code)."""
    os.makedirs(BINDIR, exist_ok=True)
    drv = os.path.join(PKG, "drivers")
    if not os.path.isdir(drv):
        return
    for name, src_name in (("test_213inplace", "test_213inplace.cu"), ("gen_ans", "gen_ans.cpp")):
        src = os.path.join(drv, src_name)
        if not os.path.exists(src):
            continue
        out = os.path.join(BINDIR, name)
        if os.path.exists(out) and os.path.getmtime(out) > max(os.path.getmtime(src), os.path.getmtime(STATIC)):
            continue
        if src.endswith(".cpp"):
            cmd = ["g++", "-O3", "-std=c++17", src, "-o", out]
        else:
            cmd = [nvcc()] + NVCC_FLAGS + [src, "-o", out, "-L" + LIBDIR, "-linplacett"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver build failed for {name}:\n{r.stdout}\n{r.stderr}")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.force))


if __name__ == "__main__":
    sys.exit(main())
