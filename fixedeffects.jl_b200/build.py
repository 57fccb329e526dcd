"""Builds libfe_b200.so (sm_100a) in-tree with nvcc.

    python fixedeffects.jl_b200/build.py [--force] [--jobs N]

Objects go to fixedeffects.jl_b200/_build/, the shared library to
fixedeffects.jl_b200/libfe_b200.so (both git-ignored; the .so travels with
the source tree to the GPU host).  The CUDA runtime is linked statically so
the library does not depend on which libcudart another module of the process
loaded.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libfe_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr", "-I", str(CSRC), "-I", str(INCLUDE)]
# the scalar recurrences round every multiply and add separately, like the
# reference's scalar code; the bulk kernels keep FMA contraction
PER_FILE = {"fe_scalar.cu": ["-fmad=false"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu"))


def _deps_mtime() -> float:
    files = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return max(f.stat().st_mtime for f in files)


def needs_build() -> bool:
    return not LIB.exists() or LIB.stat().st_mtime < _deps_mtime()


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()
    objs = []
    cmds = []
    # an object is rebuilt when its source, any header or this script is
    # newer than it (every source includes the shared headers)
    hdr = max([f.stat().st_mtime for f in list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh"))
               + list(INCLUDE.glob("*.h")) + [Path(__file__)]])
    for src in sources():
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if (not force and obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime
                and obj.stat().st_mtime >= hdr):
            continue
        cmds.append([cc, *ARCH, *COMMON, *PER_FILE.get(src.name, []), "-c", str(src), "-o", str(obj)])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        for msg in ex.map(run, cmds):
            if msg.strip() and verbose:
                print(msg, file=sys.stderr)
    tmp = LIB.with_suffix(".so.tmp")
    link = [cc, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
    run(link)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))
