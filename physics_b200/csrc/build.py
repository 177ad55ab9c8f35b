"""Build recipe of the in-tree native library (run as a script, no package import).

* ``physics_b200/lib/libphysph.so`` — the product: CUDA kernels for sm_100a,
  the C++ host mirror of the reference's fluid API and the C ABI of
  ``include/phy_ffi.h`` / ``include/phy_fluid.h``.
The library is rebuilt only when a source or header is newer than it.  The CPU
oracle (test infrastructure) has its own recipe in ``oracle/Makefile``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
PKG = ROOT / "physics_b200"
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
OBJDIR = PKG / "_build"
LIB = LIBDIR / "libphysph.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-warn-spills",
]
# Per-file flags: the f64 plain passes must not contract a*b+c into an FMA.
PER_FILE = {
    "step_plain.cu": ["-fmad=false"],
    "noalloc.cu": ["-fmad=false"],
    "grid.cu": ["-fmad=false"],
    "fluid_world.cu": ["-fmad=false"],
    "couple.cu": ["-fmad=false"],
}
SOURCES = ["grid.cu", "step_plain.cu", "step_comp.cu", "step_tiled.cu", "fluid_world.cu", "ffi.cpp",
           "checkpoint.cpp", "noalloc.cu", "adjoint.cu", "couple.cu"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _newest(paths) -> float:
    return max((p.stat().st_mtime for p in paths if p.exists()), default=0.0)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), file=sys.stderr)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, file=sys.stderr)
    return r


def build_product(force: bool = False, verbose: bool = False) -> Path:
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    srcs = [CSRC / s for s in SOURCES]
    hdr_time = _newest(headers + [Path(__file__)])
    if not force and LIB.exists() and LIB.stat().st_mtime >= max(_newest(srcs), hdr_time):
        return LIB
    OBJDIR.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for src in srcs:
        obj = OBJDIR / (src.name + ".o")
        objs.append(obj)
        if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_time):
            continue
        cmd = [nvcc, *NVCC_COMMON, *PER_FILE.get(src.name, []), "-I", ROOT / "include", "-c", src, "-o", obj]
        if src.suffix == ".cpp":
            cmd = [nvcc, "-std=c++17", "-O2", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", ROOT / "include",
                   "-x", "c++", "-c", src, "-o", obj]
        _run(cmd, verbose)
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"], verbose)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build_product(force="--force" in sys.argv, verbose=True)
