"""Airfoil contours: the NACA 4-digit formula and coordinate files, splined by arc length.

A contour runs clockwise from the trailing edge: lower surface, leading edge,
upper surface, back to the trailing edge (the orientation the generated grids
need, as ``src/jaxrans/geometry/airfoil.py:24-110`` holds it).  The leading edge
is the point farthest from the trailing-edge midpoint.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np
from scipy.interpolate import CubicSpline


@dataclass(frozen=True)
class Section:
    """Contour points ``x, y`` clockwise from the trailing edge."""

    name: str
    x: np.ndarray
    y: np.ndarray

    def __post_init__(self) -> None:
        if self.x.size < 5:
            raise ValueError(f"airfoil {self.name!r}: at least 5 points are needed, got {self.x.size}")
        if np.any(np.hypot(np.diff(self.x), np.diff(self.y)) == 0.0):
            raise ValueError(f"airfoil {self.name!r}: repeated consecutive points")

    @property
    def arc(self) -> np.ndarray:
        return np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(self.x), np.diff(self.y)))])

    @property
    def length(self) -> float:
        return float(self.arc[-1])

    @property
    def gap(self) -> float:
        return float(np.hypot(self.x[-1] - self.x[0], self.y[-1] - self.y[0]))

    @property
    def nose(self) -> int:
        mid = 0.5 * np.array([self.x[0] + self.x[-1], self.y[0] + self.y[-1]])
        return int(np.argmax(np.hypot(self.x - mid[0], self.y - mid[1])))

    @property
    def chord(self) -> float:
        mid = 0.5 * np.array([self.x[0] + self.x[-1], self.y[0] + self.y[-1]])
        k = self.nose
        return float(np.hypot(self.x[k] - mid[0], self.y[k] - mid[1]))

    @property
    def sharp(self) -> bool:
        return self.gap <= 1e-6 * self.chord

    def splines(self) -> tuple[CubicSpline, CubicSpline]:
        x, y = self.x.copy(), self.y.copy()
        if self.sharp:
            x[-1], y[-1] = x[0], y[0]
        s = self.arc
        return CubicSpline(s, x), CubicSpline(s, y)

    def at(self, s: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        fx, fy = self.splines()
        return fx(s), fy(s)

    def normalised(self) -> "Section":
        """Leading edge at the origin, chord 1, not rotated."""
        k, c = self.nose, self.chord
        return Section(self.name, (self.x - self.x[k]) / c, (self.y - self.y[k]) / c)


def clockwise(x, y, name: str) -> Section:
    """Points round a contour in either direction, from either trailing-edge end,
    reordered clockwise from the trailing edge."""
    x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
    keep = np.concatenate([[True], np.hypot(np.diff(x), np.diff(y)) > 0.0])
    x, y = x[keep], y[keep]
    signed = 0.5 * (np.sum(x[:-1] * y[1:] - x[1:] * y[:-1]) + (x[-1] * y[0] - x[0] * y[-1]))
    if signed > 0.0:
        x, y = x[::-1], y[::-1]
    return Section(name, x, y)


def naca4(code: str, n: int = 201, sharp: bool = True) -> Section:
    """NACA 4-digit section (Abbott & von Doenhoff, *Theory of Wing Sections*,
    6.4): thickness ``t`` over a camber line of maximum ``m`` at ``p``, cosine
    spaced, ``2 n - 1`` points; ``sharp`` uses the closed trailing-edge
    coefficient -0.1036 in place of -0.1015."""
    if len(code) != 4 or not code.isdigit():
        raise ValueError(f"a NACA 4-digit code is four digits, got {code!r}")
    m, p, t = int(code[0]) / 100.0, int(code[1]) / 10.0, int(code[2:]) / 100.0
    xc = 0.5 * (1.0 - np.cos(np.linspace(0.0, np.pi, n)))
    last = -0.1036 if sharp else -0.1015
    half = 5.0 * t * (0.2969 * np.sqrt(xc) - 0.1260 * xc - 0.3516 * xc ** 2 + 0.2843 * xc ** 3 + last * xc ** 4)
    if m > 0.0 and p > 0.0:
        fore = xc < p
        camber = np.where(fore, m / p ** 2 * (2 * p * xc - xc ** 2),
                          m / (1 - p) ** 2 * (1 - 2 * p + 2 * p * xc - xc ** 2))
        slope = np.where(fore, 2 * m / p ** 2 * (p - xc), 2 * m / (1 - p) ** 2 * (p - xc))
    else:
        camber, slope = np.zeros_like(xc), np.zeros_like(xc)
    theta = np.arctan(slope)
    xu, yu = xc - half * np.sin(theta), camber + half * np.cos(theta)
    xl, yl = xc + half * np.sin(theta), camber - half * np.cos(theta)
    x = np.concatenate([xl[::-1], xu[1:]])
    y = np.concatenate([yl[::-1], yu[1:]])
    if sharp:
        y[0] = y[-1] = 0.5 * (y[0] + y[-1])
    return clockwise(x, y, f"NACA {code}")


def read_coordinates(path: str | Path) -> Section:
    """A Selig (name line, then the points round the contour), Lednicer (name,
    point counts, upper then lower from the leading edge) or two-column file."""
    path = Path(path)
    rows, name = [], path.stem
    for line in path.read_text().splitlines():
        parts = line.replace(",", " ").split()
        try:
            values = [float(v) for v in parts]
        except ValueError:
            if not rows and parts:
                name = line.strip()
            continue
        if len(values) == 2:
            rows.append(values)
    data = np.array(rows)
    if len(data) < 5:
        raise ValueError(f"{path.name}: fewer than 5 coordinate pairs")
    if data[0, 0] > 1.5 and data[0, 1] > 1.5:
        nu, nl = int(data[0, 0]), int(data[0, 1])
        upper, lower = data[1:1 + nu], data[1 + nu:1 + nu + nl]
        contour = np.concatenate([upper[::-1], lower[1:]])
        return clockwise(contour[:, 0], contour[:, 1], name)
    return clockwise(data[:, 0], data[:, 1], name)


def section_source(spec: str, base: Path | None = None) -> Section:
    """``naca####`` (``naca####_blunt`` for the open trailing edge), else a file."""
    low = spec.lower()
    if low.startswith("naca") and low[4:8].isdigit() and len(low) in (8, 14):
        return naca4(low[4:8], sharp=not low.endswith("_blunt"))
    for root in ([base] if base else []) + [Path.cwd()]:
        path = Path(spec) if Path(spec).is_absolute() else root / spec
        if path.is_file():
            return read_coordinates(path)
    raise FileNotFoundError(f"airfoil {spec!r}: not a NACA 4-digit name, nor a file")
