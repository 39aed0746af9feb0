"""Build libn_body_sim_pro_cuda.so in-tree (n_body_sim_pro_b200/lib/).

CUDA sources are compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); the C17 host layer by gcc.
The result links the CUDA runtime statically and exports only the symbols
declared in include/n_body_sim_pro_cuda.h.  Incremental: a translation unit
is rebuilt when it or any header of csrc/ or include/ is newer than its object.

    python -m n_body_sim_pro_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libn_body_sim_pro_cuda.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                     "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + INCLUDE]
# presets.cu follows the reference's FP64 generation formulas, which are
# compiled without FMA: no contraction there.
FILE_FLAGS = {"presets.cu": ["--fmad=false"]}
CC_FLAGS = ["-O2", "-std=c17", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wextra",
            "-Wno-unused-parameter", "-I" + CSRC, "-I" + INCLUDE]


def _cuda_home() -> str:
    for cand in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if cand and os.path.exists(os.path.join(cand, "bin", "nvcc")):
            return cand
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(nvcc))
    raise RuntimeError("nvcc not found: set CUDA_HOME")


def _cc() -> str:
    # The system gcc; an inherited CC may point at a toolchain without the
    # standard library layout nvcc expects.
    return "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else (shutil.which("gcc") or "cc")


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj: str, src: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> str:
    cuda = _cuda_home()
    nvcc = os.path.join(cuda, "bin", "nvcc")
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    deps = _headers()
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            extra = FILE_FLAGS.get(os.path.basename(src), [])
            _run([nvcc, "-ccbin", _cc()] + NVCC_FLAGS + extra + ["-c", src, "-o", obj], verbose)
    for src in sorted(glob.glob(os.path.join(CSRC, "*.c"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            _run([_cc()] + CC_FLAGS + ["-I" + os.path.join(cuda, "include"), "-c", src, "-o", obj],
                 verbose)
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB)
                                                for o in objs):
        tmp = LIB + ".tmp"
        _run([nvcc, "-ccbin", _cc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs +
             ["-Xlinker", "--exclude-libs,ALL"], verbose)
        os.replace(tmp, LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
