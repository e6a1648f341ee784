"""Build recipe of the native library (librrg.so) and the `rrgsim` executable.

Everything is compiled in-tree for sm_100a with nvcc:
  rrgsim_b200/_build/*.o   objects (git-ignored)
  rrgsim_b200/librrg.so    the C-ABI library (include/rrg.h)
  rrgsim_b200/bin/rrgsim   the solver executable, linked against librrg.so

`python -m rrgsim_b200.build` rebuilds what is out of date.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "librrg.so"
BIN = PKG / "bin" / "rrgsim"
INCLUDE = ROOT / "include"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                  "-I", str(INCLUDE), "-I", str(CSRC), "--expt-relaxed-constexpr"]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-I", str(INCLUDE), "-I",
            str(CSRC), "-I", "/usr/local/cuda/include"]

LIB_SOURCES = ["direct.cu", "integrate.cu", "pm.cu", "context.cu", "adjoint.cu", "host_io.cpp",
               "run.cpp", "noalloc.cu", "sort.cu", "ensemble.cu", "pm_adjoint.cu",
               "wave_solve.cu"]


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "rrg.h"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not _stale(obj, [src] + _headers()):
        return obj
    if src.suffix == ".cu":
        cmd = [NVCC] + CUFLAGS + ["-c", str(src), "-o", str(obj)]
    else:
        cmd = [NVCC, "-x", "c++", "-Xcompiler", ",".join(CXXFLAGS[:1] + ["-fPIC", "-fvisibility=hidden"]),
               "-std=c++17", "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compiles librrg.so and bin/rrgsim if out of date; returns the library path."""
    BUILD.mkdir(exist_ok=True)
    BIN.parent.mkdir(exist_ok=True)
    if force:
        for o in BUILD.glob("*.o"):
            o.unlink()
    srcs = [CSRC / s for s in LIB_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + \
              ["-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    cli = CSRC / "rrgsim_cli.cpp"
    if _stale(BIN, [cli, LIB, INCLUDE / "rrg.h"]):
        cmd = ["g++", "-O2", "-std=c++17", "-I", str(INCLUDE), str(cli), "-o", str(BIN),
               "-L", str(PKG), "-lrrg", "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"rrgsim link failed\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
