"""Builds the in-tree CUDA library hadros_b200/lib/libhadros_b200.so for sm_100a.

    python -m hadros_b200.build          # incremental
    python -m hadros_b200.build --force  # rebuild everything

The reference-arithmetic trace kernel is compiled with --fmad=false (no
contraction of a*b+c into an FMA) so that its FP64 arithmetic rounds like the
reference's x86-64 build; the fast-geodesic variant is compiled with FMA.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
BUILD_DIR = PKG / "_build"
LIB = LIB_DIR / "libhadros_b200.so"
BIN_DIR = PKG / "bin"
CLI = BIN_DIR / "compute_kerr_image"
REPO = PKG.parent
INCLUDE = REPO / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra"]

# (source, extra nvcc flags): the reference-arithmetic kernel must not contract
# a*b+c into FMAs; the fast-geodesic kernel does.
CU_SOURCES = [("hadros_trace.cu", ["--fmad=false"]), ("hadros_trace_fast.cu", ["--fmad=true"]),
              ("hadros_noalloc.cu", ["--fmad=false"]), ("hadros_mlp.cu", []), ("hadros_mlp_umma.cu", [])]
CXX_SOURCES = ["hadros_host.cpp", "hadros_formats.cpp"]
HEADERS = ["hadros_internal.h", "hadros_physics.cuh", "hadros_physics_f32.cuh", "hadros_mev.cuh",
           "hadros_trace_kernel.cuh", "hadros_mlp.cuh", "hadros_umma.cuh",
           "hadros_cr_math.cuh", "hadros_sincos_table.h"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the hadros_b200 CUDA library cannot be built")


def _cuda_home() -> Path:
    return Path(_nvcc()).resolve().parent.parent


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], log: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    log.append(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the CUDA kernels and the C-ABI host code; returns the .so path."""
    BUILD_DIR.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    nvcc = _nvcc()
    cuda_inc = _cuda_home() / "include"
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "hadros_b200.h"]
    objs: list[Path] = []
    log: list[str] = []
    for src, extra in CU_SOURCES:
        obj = BUILD_DIR / (Path(src).stem + ".o")
        if force or _stale(obj, [CSRC / src] + headers):
            _run([nvcc, *ARCH, *NVCC_FLAGS, *extra, "-I", str(INCLUDE), "-c", str(CSRC / src),
                  "-o", str(obj)], log, verbose)
        objs.append(obj)
    for src in CXX_SOURCES:
        obj = BUILD_DIR / (Path(src).stem + ".o")
        if force or _stale(obj, [CSRC / src] + headers):
            _run(["g++", *CXX_FLAGS, "-I", str(INCLUDE), "-I", str(cuda_inc), "-c",
                  str(CSRC / src), "-o", str(obj)], log, verbose)
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fPIC",
              "-o", str(LIB), *map(str, objs)], log, verbose)
    BIN_DIR.mkdir(exist_ok=True)
    main_src = CSRC / "compute_kerr_image_main.cpp"
    if force or _stale(CLI, [main_src, LIB, INCLUDE / "hadros_b200.h"]):
        _run(["g++", *CXX_FLAGS, "-I", str(INCLUDE), "-o", str(CLI), str(main_src),
              "-L", str(LIB_DIR), "-lhadros_b200", "-Wl,-rpath,$ORIGIN/../lib"], log, verbose)
    (BUILD_DIR / "build.log").write_text("\n".join(log))
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
