"""Shared test set-up: import paths, the ``gpu`` marker."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "jax-rans_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: long-running")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(scope="session", autouse=True)
def fresh_library(request):
    """The C-ABI library rebuilt in place when a source is newer (nvcc is on the GPU box too)."""
    if any(item.get_closest_marker("gpu") for item in request.session.items) and gpu_available():
        from jaxrans_b200.build import build
        build()


@pytest.fixture(scope="session")
def harness(tmp_path_factory):
    """The 3D kernels' host-and-device bodies built for the host (tests/host3d/harness.cu,
    nvcc with no device code): the 3D kernels' arithmetic run without a GPU."""
    import ctypes as C
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc is not available")
    out = tmp_path_factory.mktemp("host3d") / "libjr3host.so"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared",
                    "-gencode", "arch=compute_100a,code=compute_100a", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "host3d" / "harness.cu"), "-o", str(out)], check=True)
    lib = C.CDLL(str(out))
    p, i, d = C.c_void_p, C.c_int, C.c_double
    for name, args in {"jr3_host_eval": [p, p, p, p, i],
                       "jr3_host_eval_faces": [p, p, p, p, i],
                       "jr3_host_wave_speeds": [p, p, p],
                       "jr3_host_precondition": [p, p, d, p, p],
                       "jr3_host_newton_steps": [p, p, p, p, p, p, i, p],
                       "jr3_host_forces": [p, p, d, d, p, p],
                       "jr3_host_wall_loads": [p, p, p],
                       "jr3_host_fill": [p, p, p, i],
                       "jr3_host_wall_distance": [p, C.c_longlong, p, i, p, i]}.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = C.c_int, args
    return lib
