"""Builds the gtomrln CUDA library in-tree for sm_100a.

    python -m gtom_b200.build          # -> gtom_b200/lib/libgtomrln.so

Every translation unit under gtom_b200/csrc/ is compiled by nvcc for
sm_100a only (``-gencode arch=compute_100a,code=sm_100a``) and linked with
cuFFT into one shared library whose exported symbols are exactly the C ABI
of include/gtomrln.h.  Objects go to gtom_b200/_build/, rebuilt when a
source or header is newer.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libgtomrln.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
           "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda) / "bin" / "nvcc"
    return str(cand) if cand.exists() else "nvcc"


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compiles and links the library; returns its path."""
    OBJ.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    heads = _headers()
    nvcc = _nvcc()
    jobs = []
    for src in srcs:
        obj = OBJ / (src.stem + ".o")
        if force or ptxas_info or _stale(obj, [src, *heads]):
            cmd = [nvcc, *ARCH, *NVFLAGS, "-c", str(src), "-o", str(obj)]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(lambda c: _run(c, verbose or ptxas_info), jobs))
    objs = [OBJ / (s.stem + ".o") for s in srcs]
    if force or jobs or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcufft"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
