"""Build recipe of the native library: every C++ / CUDA source of hsolve_b200/csrc is compiled for
sm_100a with nvcc into hsolve_b200/lib/libhsolve_b200.so (in-tree, so it ships with the package).

    python -m hsolve_b200.build [-v] [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC = PKG / "csrc"
INC = PKG.parent / "include"
LIB = PKG / "lib"
OBJ = LIB / "obj"
SO = LIB / "libhsolve_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          f"-I{INC}", f"-I{SRC}"]


def _sources():
    return sorted(p for p in SRC.iterdir() if p.suffix in (".cu", ".cpp") and not p.name.startswith("py"))


def _headers_mtime() -> float:
    hs = [p for p in SRC.iterdir() if p.suffix in (".hpp", ".cuh", ".h")] + list(INC.glob("*.h"))
    return max((p.stat().st_mtime for p in hs), default=0.0)


def _compile(src: Path, force: bool, verbose: bool) -> Path:
    obj = OBJ / (src.stem + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, _headers_mtime()):
        return obj
    cmd = [NVCC, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd.insert(1, "-Xptxas=-v" if verbose else "-Xptxas=-O3")
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    if force or not SO.exists() or SO.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(SO), *map(str, objs), "-lcudart", "-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return SO


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(SO)
