"""Builds the in-tree shared library libtdmd_b200.so for sm_100a with nvcc.

The library is plain CUDA C++ behind the C ABI in include/tdmd_b200.h; no
torch headers are involved, so it is a direct nvcc -shared build (one object
per translation unit, compiled in parallel, relinked only when a source or
header changed).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libtdmd_b200.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max(os.path.getmtime(h) for h in hs)


def _compile(src, hdr_mtime, verbose):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
        return obj, False
    cmd = [NVCC, *ARCH, *FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stderr)
    return obj, True


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr = _headers_mtime()
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, hdr, verbose), srcs))
    objs = [o for o, _ in results]
    changed = any(c for _, c in results)
    if changed or not os.path.exists(LIB):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_driver()
    return LIB


DRIVER_SRC = os.path.join(PKG, "driver", "tdmd_standalone.cpp")
DRIVER_DIR = os.path.join(PKG, "bin", "native")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_driver() -> dict:
    """The native tdmd_standalone, once per precision as the reference builds
    it (bin/native/tdmd_standalone: FP64, bin/native/tdmd_standalone_mixed),
    compiled with the host C++ compiler against include/tdmd_b200.hpp and
    linked to the library (rpath relative to the binary)."""
    os.makedirs(DRIVER_DIR, exist_ok=True)
    gxx = os.environ.get("CXX", "g++")
    deps = max(os.path.getmtime(DRIVER_SRC), _headers_mtime(), os.path.getmtime(LIB))
    out = {}
    for name, define in (("tdmd_standalone", "TDMD_PRECISION_FP64"),
                         ("tdmd_standalone_mixed", "TDMD_PRECISION_MIXED")):
        exe = os.path.join(DRIVER_DIR, name)
        out[name] = exe
        if os.path.exists(exe) and os.path.getmtime(exe) >= deps:
            continue
        cmd = [gxx, "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", f"-D{define}=1",
               "-I", INCLUDE, "-I", os.path.join(CUDA_HOME, "include"), DRIVER_SRC, "-o", exe,
               LIB, "-Wl,-rpath,$ORIGIN/../.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
