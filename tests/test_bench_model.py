"""The benchmark's byte model and roofline arithmetic (bench.py), on the host: the
algorithmic bytes per cell each roofline divides by, and the achieved bandwidth and
fraction it reports from a kernel's CUDA-event time."""

from __future__ import annotations

import pytest

import bench


def test_jv_tile_bytes_per_cell():
    # SA: 2 faces x 68 coefficients and 7 cell coefficients, U, v, out (5 each), V/dt, the
    # centre (2), the volume and four face components -- FP64
    assert bench.jvp_bytes_per_cell("sa", 5) == 8 * (2 * 68 + 7 + 15 + 1 + 2 + 1 + 4) == 1328
    # the mixed form stores the face coefficients in FP32
    assert bench.jvp_bytes_per_cell("sa", 5, fp32_faces=True) == 1328 - 4 * 2 * 68 == 784
    assert bench.jvp_bytes_per_cell("euler", 4) == 8 * (2 * 32 + 12 + 1)
    assert bench.jvp_bytes_per_cell("laminar", 4) == 8 * (2 * 51 + 12 + 1 + 2)


def test_residual_and_3d_bytes_per_cell():
    assert bench.residual_bytes_per_cell("sa", 5) == 144
    assert bench.residual_bytes_per_cell("euler", 4) == 8 * (8 + 1 + 4)
    assert bench.jvp3d_bytes_per_cell(6) == 256


def test_roofline_arithmetic():
    peaks = {"hbm_gbs": 6400.0, "source": "measured"}
    kern = {"jvp_tile": 0.0185, "residual_tile": 0.0206}
    r = bench.roofline_of(kern, "sa", 5, 36864, peaks)
    assert r["algorithmic_bytes_per_launch"] == 1328 * 36864
    assert r["achieved"] == pytest.approx(1328 * 36864 / 18.5e-6 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 6400.0)
    res = bench.roofline_of(kern, "sa", 5, 36864, peaks, kernel="residual_tile")
    assert res["algorithmic_bytes_per_cell"] == 144 and res["launch_ms"] == 0.0206
    mixed = bench.roofline_of(kern, "sa", 5, 36864, peaks, fp32_faces=True)
    assert mixed["algorithmic_bytes_per_cell"] == 784


def test_whole_job_rate_counts_every_rank():
    # 3 solves of 2 cases on each of 4 ranks in 36 s: 24 solves in 36 s
    assert bench.whole_job_rate(3, 2, 4, 36.0) == pytest.approx(3600.0 * 24 / 36.0)
