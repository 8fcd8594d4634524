"""Build libumapb200.so in-tree with nvcc for sm_100a.

Usage: python -m umapers_b200.build [--force]

Every .cu / .cpp file under csrc/ is compiled to an object under
umapers_b200/_build/ and linked into umapers_b200/libumapb200.so.  CUDA code
is generated for sm_100a only (`-gencode arch=compute_100a,code=sm_100a`).
Host files are compiled with -ffp-contract=off so host arithmetic rounds as
the reference's Rust build does.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libumapb200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "--extended-lambda",
    "-ccbin",
    HOST_CXX,
    "-Xcompiler",
    "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    "-Xptxas",
    "-v",
] + ARCH


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list((PKG.parent / "include").glob("*.h")))


def _needs(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    newest = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    return obj.stat().st_mtime < newest


def _compile(src: Path, force: bool) -> tuple[Path, str]:
    obj = BUILD / (src.name + ".o")
    if not force and not _needs(obj, src):
        return obj, ""
    if src.suffix == ".cu":
        cmd = [NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = [HOST_CXX, "-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fvisibility=hidden",
               "-I/usr/local/cuda/include", "-c", str(src), "-o", str(obj)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    return obj, proc.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    objs = [r[0] for r in results]
    if verbose:
        for _, log in results:
            if log:
                print(log)
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [NVCC, "-shared", *ARCH, "-ccbin", HOST_CXX, "-o", str(LIB), *map(str, objs),
               "-Xlinker", "--exclude-libs,ALL", "-lpthread"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
