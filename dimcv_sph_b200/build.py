"""Builds libdimcv.so (sm_100a) in-tree with nvcc.

The SPH translation units are compiled with ``-fmad=false`` (no FMA
contraction) and IEEE division / square root so that every per-pair
expression rounds exactly as written; the N-body unit (dv_vvpe.cu) keeps FMA
contraction on.  Objects go to ``dimcv_sph_b200/_build``; the shared library
lands next to this file so that it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libdimcv.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler",
          "-fvisibility=hidden", "--expt-relaxed-constexpr", f"-I{INCLUDE}"]
# unit -> extra flags
UNITS = {
    "dv_capi.cu": ["-fmad=false"],
    "dv_grid.cu": ["-fmad=false"],
    "dv_sph.cu": ["-fmad=false"],
    "dv_dimcv.cu": ["-fmad=false"],
    "dv_vvpe.cu": [],
    "dv_noalloc.cu": ["-fmad=false"],
    "dv_vpm.cu": [],
    "dv_batch.cu": ["-fmad=false"],
}


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libdimcv")
    return exe


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compiles every unit that changed and links libdimcv.so; returns its path."""
    BUILD.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + [INCLUDE / "dimcv.h"]
    objs = []
    for unit, extra in UNITS.items():
        src = CSRC / unit
        obj = BUILD / (unit + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, *headers, Path(__file__)]):
            cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {unit}:\n{r.stdout}\n{r.stderr}")
            if ptxas_verbose or verbose:
                sys.stderr.write(r.stderr)
    if force or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
