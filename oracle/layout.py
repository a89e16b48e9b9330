"""Real row-normalized KB interpolation of the reference layout oracle (restated).

TEST INFRASTRUCTURE: see oracle/__init__.py.

``generate_trajectory`` follows src/nufft_layout_oracle.py:124-149 and
``build_interpolation`` follows :159-206 (separable KB weights of :152-156,
non-periodic support, row sums normalized to one, columns sorted).  These feed
the export-format goldens (src/export_gpu_case.py:171-181).
"""
from __future__ import annotations

import math

import numpy as np

from . import planner as P


def generate_trajectory(kind: str, grid_size: int, n_samples: int) -> np.ndarray:
    center = (grid_size - 1) / 2.0
    rmax = 0.43 * grid_size
    if kind == "radial":
        spokes = max(16, int(round(math.sqrt(n_samples))))
        per = int(math.ceil(n_samples / spokes))
        golden = math.pi * (3.0 - math.sqrt(5.0))
        radii = np.linspace(-rmax, rmax, per, endpoint=True)
        pts = []
        for s in range(spokes):
            a = s * golden
            ca, sa = math.cos(a), math.sin(a)
            for r in radii:
                pts.append((center + r * ca, center + r * sa))
        return np.asarray(pts[:n_samples], dtype=np.float64)
    if kind == "spiral":
        t = (np.arange(n_samples, dtype=np.float64) + 0.5) / n_samples
        turns = max(6.0, grid_size / 8.0)
        radius = rmax * np.sqrt(t)
        angle = 2.0 * math.pi * turns * t
        return np.column_stack((center + radius * np.cos(angle), center + radius * np.sin(angle)))
    raise ValueError(kind)


def _weight(d: float, width: int, beta: float) -> float:
    s = 2.0 * d / width
    if abs(s) >= 1.0:
        return 0.0
    return float(np.i0(beta * math.sqrt(max(0.0, 1.0 - s * s))) / np.i0(beta))


def build_interpolation(traj: np.ndarray, grid_size: int, width: int, oversampling: float = 2.0) -> P.View:
    beta = math.pi * math.sqrt(max((width / oversampling * (oversampling - 0.5)) ** 2 - 0.8, 0.01))
    half = width // 2
    cols, vals = [], []
    for x, y in traj:
        xs = int(math.floor(x)) - half + 1
        ys = int(math.floor(y)) - half + 1
        ent = []
        for gy in range(ys, ys + width):
            if gy < 0 or gy >= grid_size:
                continue
            wy = _weight(y - gy, width, beta)
            for gx in range(xs, xs + width):
                if gx < 0 or gx >= grid_size:
                    continue
                v = _weight(x - gx, width, beta) * wy
                if v != 0.0:
                    ent.append((gy * grid_size + gx, v))
        norm = sum(v for _, v in ent)
        ent.sort(key=lambda e: e[0])
        cols.append([c for c, _ in ent])
        vals.append([v / norm for _, v in ent])
    m = len(traj)
    return P.View(np.arange(m, dtype=np.int64), cols, vals, np.asarray(traj, dtype=np.float64), m,
                  grid_size * grid_size)


def build_view(spec: dict) -> P.View:
    traj = generate_trajectory(spec["trajectory"], spec["grid"], spec["samples"])
    fwd = build_interpolation(traj, spec["grid"], spec["width"])
    return P.transpose(fwd, spec["grid"]) if spec["view"] == "G_T" else fwd
