"""Build the sm_100a shared library ``libevd_b200.so`` (and the ``myEVD`` CLI).

Every ``csrc/*.cu`` file is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` into an object
under ``_build/`` and linked into ``evd4sc2025_b200/libevd_b200.so`` next to
this file (in-tree, so it travels with the source tree).
``cli/myEVD.cu`` is linked against it into ``evd4sc2025_b200/bin/myEVD``.

Usage: ``python -m evd4sc2025_b200.build [-j N] [--force]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libevd_b200.so"
BIN = PKG / "bin" / "myEVD"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
              "--expt-relaxed-constexpr", "-I", str(INCLUDE)]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build evd_b200")


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: pathlib.Path, force: bool) -> pathlib.Path:
    obj = BUILD / (src.stem + ".o")
    if (not force and obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime
            and obj.stat().st_mtime >= _headers_mtime()):
        return obj
    cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(jobs: int = 8, force: bool = False, verbose: bool = False) -> pathlib.Path:
    """Compile and link; returns the path of the shared library."""
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        if verbose:
            print(f"linked {LIB}")
    cli_src = PKG / "cli" / "myEVD.cu"
    if cli_src.exists():
        BIN.parent.mkdir(exist_ok=True)
        if force or not BIN.exists() or BIN.stat().st_mtime < max(
                LIB.stat().st_mtime, cli_src.stat().st_mtime):
            cmd = [_nvcc(), *ARCH, "-O2", "-std=c++17", "-I", str(INCLUDE), str(cli_src),
                   "-o", str(BIN), "-L", str(PKG), "-levd_b200",
                   "-Xlinker", "-rpath,$ORIGIN/.."]
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode != 0:
                raise RuntimeError(f"myEVD link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("-j", "--jobs", type=int, default=8)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    path = build(args.jobs, args.force, verbose=True)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
