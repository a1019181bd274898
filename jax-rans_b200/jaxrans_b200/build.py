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


FFI_SOURCE = CSRC / "ffi" / "jr_ffi.cc"
FFI_LIB = PKG / "lib" / "libjaxrans_b200_ffi.so"


def ffi_include_dir() -> str | None:
    """JAX's XLA FFI header directory, or None where JAX is not installed."""
    try:
        import jax.ffi
    except ImportError:
        return None
    return jax.ffi.include_dir()


def build_ffi(force: bool = False) -> Path | None:
    """Compile the jax.ffi handlers (``csrc/ffi/jr_ffi.cc``) against JAX's FFI headers,
    linked to the library.  Returns None, building nothing, where JAX is absent."""
    include = ffi_include_dir()
    if include is None:
        return None
    lib = build()
    if not force and FFI_LIB.is_file() and FFI_LIB.stat().st_mtime > max(FFI_SOURCE.stat().st_mtime,
                                                                         lib.stat().st_mtime):
        return FFI_LIB
    cuda = Path(nvcc()).resolve().parents[1]
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", f"-I{include}", f"-I{INCLUDE}", f"-I{cuda / 'include'}",
           str(FFI_SOURCE), f"-L{lib.parent}", "-ljaxrans_b200", f"-Wl,-rpath,{lib.parent}", f"-L{cuda / 'lib64'}",
           "-lcudart", "-o", str(FFI_LIB)]
    subprocess.run(cmd, check=True)
    return FFI_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    if "--ffi" in sys.argv:
        print(build_ffi(force="--force" in sys.argv) or "JAX is not installed: the jax.ffi handlers are not built")
