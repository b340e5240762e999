"""Builds libwarpsolve.so in-tree for sm_100a with nvcc (no JIT cache, no pip install).

The library is the product: the C ABI declared in include/warpsolve.h.  Each
translation unit compiles in parallel; the link step produces
starhub_b200/libwarpsolve.so next to this file.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libwarpsolve.so"
SOURCES = ["ws_api.cu", "ws_index.cu", "ws_solve.cu", "ws_graph.cu", "ws_server.cu", "ws_measure.cu"]
# The measurement maps keep every multiply and add separately rounded, as the host restatement
# of their eigen solver does: its branches test quantities against the FP32 epsilon.
FILE_FLAGS = {"ws_measure.cu": ["--fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-Xcompiler", "-pthread",
         "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libwarpsolve.so")


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "warpsolve.h"]
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()
    jobs = []
    for s in SOURCES:
        src = CSRC / s
        obj = BUILD / (s + ".o")
        if force or _stale(obj, src):
            jobs.append([cc, *ARCH, *FLAGS, *FILE_FLAGS.get(s, []), "-c", str(src), "-o", str(obj)])
    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, file=sys.stderr)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        list(ex.map(run, jobs))
    objs = [str(BUILD / (s + ".o")) for s in SOURCES]
    if force or jobs or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        run([cc, *ARCH, "-shared", "--cudart", "static", "-Xcompiler", "-pthread", "-o", str(tmp), *objs])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
