"""Build the C-ABI library in place: ``python -m jaxrans_b200.build``.

One ``nvcc`` call compiles the sm_100a kernels and the C ABI into
``jaxrans_b200/lib/libjaxrans_b200.so``; it is rebuilt only when a source is newer.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG.parent / "csrc"
INCLUDE = PKG.parents[1] / "include"
SOURCES = ("residual.cu", "linesolve.cu", "krylov.cu", "forces.cu", "capi.cu", "residual3d.cu", "linesolve3d.cu", "newton3d.cu", "walldist3d.cu", "capi3d.cu")
LIB = PKG / "lib" / "libjaxrans_b200.so"
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).is_file():
            return cand
    raise FileNotFoundError("nvcc not found (set NVCC)")


def stale() -> bool:
    if not LIB.is_file():
        return True
    built = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [INCLUDE / "jaxrans_b200.h"]
    return any(d.stat().st_mtime > built for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           f"-I{INCLUDE}", *(str(CSRC / s) for s in SOURCES), "-o", str(tmp)]
    if verbose:
        cmd.insert(2, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
