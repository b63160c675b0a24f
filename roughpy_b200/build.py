"""Build the sm_100a shared library ``librpyb.so`` in-tree.

``python roughpy_b200/build.py`` compiles every source under ``csrc/`` with
nvcc for ``sm_100a`` only and links ``roughpy_b200/_lib/librpyb.so``.  Object
files go to ``_build/`` at the repository root and are rebuilt only when a
source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "librpyb.so"
BUILD = ROOT / "_build" / "rpyb"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I", str(ROOT / "include"),
]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = pathlib.Path(cuda) / "bin" / "nvcc"
    if cand.exists():
        return str(cand)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found; set CUDA_HOME")
    return found


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers():
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "rpyb.h"]


def _stale(target: pathlib.Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: pathlib.Path, verbose: bool) -> pathlib.Path:
    obj = BUILD / (src.name + ".o")
    if not _stale(obj, [src] + _headers()):
        return obj
    cmd = [_nvcc()] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [_nvcc(), "-x", "cu"] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> pathlib.Path:
    """Compile (if needed) and return the path of ``librpyb.so``."""
    BUILD.mkdir(parents=True, exist_ok=True)
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + [
            "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
