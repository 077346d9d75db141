"""Build recipe of libsolvix_b200.so (sm_100a only).

Compiles every ``csrc/*.cu`` with nvcc for ``compute_100a/sm_100a`` and the
host ``csrc/*.cpp`` with g++, then links one shared library in-tree
(``solvix_b200/libsolvix_b200.so``) against the static CUDA runtime.  The
element / stress translation unit is compiled with ``-fmad=false`` so that
its arithmetic rounds operation by operation, like the reference's Rust.
Objects go to ``solvix_b200/_build/``; a unit is recompiled when its source
or any header is newer than its object.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libsolvix_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = shutil.which("nvcc") or os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                     "-Xptxas", "-warn-spills", f"-I{INCLUDE}", f"-I{CSRC}"]
# units whose arithmetic must round like the reference (no fused multiply-add)
NO_FMA = {"svx_element.cu"}
CXX = os.environ.get("CXX", "g++")
# host arithmetic that restates the reference's (load vectors) must round
# operation by operation: Rust never fuses a*b+c
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra",
             f"-I{INCLUDE}", f"-I{CSRC}",
             f"-I{os.path.join(CUDA_HOME, 'include')}"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj: str, src: str, headers) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src, *headers])


def _compile(src: str, verbose: bool) -> str:
    name = os.path.basename(src)
    obj = os.path.join(BUILD, name + ".o")
    if src.endswith(".cu"):
        cmd = [NVCC, *NVCC_FLAGS]
        if name in NO_FMA:
            cmd.append("-fmad=false")
        cmd += ["-c", src, "-o", obj]
    else:
        cmd = [CXX, *CXX_FLAGS, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {name} failed:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stderr.strip() or r.stdout.strip()):
        print(r.stdout + r.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile (incrementally) and link the library; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    objs = [os.path.join(BUILD, os.path.basename(s) + ".o") for s in srcs]
    todo = [s for s, o in zip(srcs, objs) if force or _stale(o, s, headers)]
    if todo:
        with ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            list(ex.map(lambda s: _compile(s, verbose), todo))
    if force or todo or not os.path.exists(LIB) or \
            any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-cudart", "static",
               "-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
