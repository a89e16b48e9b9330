"""Seeded synthetic inputs: phantoms, coil maps, trajectories, density weights.

The reference measures on OCMR (a public dataset that is not available here);
these generators stand in for it with the shapes and value distributions of
the benchmark configurations:

* random-ellipse phantom, magnitudes U(0.1, 1), smooth linear-ramp phase
* Gaussian-blob complex coil sensitivities, centres evenly on a circle of
  radius 0.7 FOV, sigma 0.4 FOV, random linear phase, root-sum-of-squares 1
* golden-angle radial trajectories in cycles/pixel in [-0.5, 0.5), built like
  experiments/data_prep/generate_trajectories.py:14-23 (golden angle
  pi*(3-sqrt(5)), readout linspace(-0.5, 0.5, endpoint=False))
* variable-density spirals (interleaves x samples, density exponent)
* ramp density compensation

Everything is numpy, FP64 internally, returned as complex64 / float32 arrays in
the reference's runtime-file layouts (coil-major ``[C][N][N]``, ``[M][2]``).
"""

from __future__ import annotations

import math

import numpy as np

BASE_SEED = 20260823


def _grid(n: int) -> tuple[np.ndarray, np.ndarray]:
    coords = (np.arange(n, dtype=np.float64) - n // 2) / n
    return np.meshgrid(coords, coords, indexing="ij")


def ellipse_phantom(n: int, seed: int, ellipses: int = 10) -> np.ndarray:
    """[N, N] complex64 phantom: sum of random ellipses times a linear-ramp phase."""
    rng = np.random.default_rng(seed)
    y, x = _grid(n)
    image = np.zeros((n, n), dtype=np.float64)
    for _ in range(ellipses):
        cy, cx = rng.uniform(-0.25, 0.25, size=2)
        ay, ax = rng.uniform(0.05, 0.3, size=2)
        theta = rng.uniform(0.0, math.pi)
        mag = rng.uniform(0.1, 1.0)
        ct, st = math.cos(theta), math.sin(theta)
        yr = (y - cy) * ct + (x - cx) * st
        xr = -(y - cy) * st + (x - cx) * ct
        image += mag * (((yr / ay) ** 2 + (xr / ax) ** 2) <= 1.0)
    slope = rng.uniform(-1.0, 1.0, size=2)
    phase = np.exp(1j * math.pi * (slope[0] * y + slope[1] * x))
    return (image * phase).astype(np.complex64)


def coil_maps(n: int, coils: int, seed: int) -> np.ndarray:
    """[C, N, N] complex64 Gaussian-blob sensitivities with RSS = 1."""
    rng = np.random.default_rng(seed + 7919)
    y, x = _grid(n)
    maps = np.zeros((coils, n, n), dtype=np.complex128)
    for c in range(coils):
        ang = 2.0 * math.pi * c / coils
        cy, cx = 0.7 * math.sin(ang), 0.7 * math.cos(ang)
        blob = np.exp(-((y - cy) ** 2 + (x - cx) ** 2) / (2.0 * 0.4 ** 2))
        slope = rng.uniform(-1.0, 1.0, size=2)
        maps[c] = blob * np.exp(1j * math.pi * (slope[0] * y + slope[1] * x))
    rss = np.sqrt(np.sum(np.abs(maps) ** 2, axis=0))
    return (maps / rss).astype(np.complex64)


def golden_radial(spokes: int, readout: int) -> np.ndarray:
    """[spokes*readout, 2] float32 golden-angle radial trajectory (cycles/pixel)."""
    golden = math.pi * (3.0 - math.sqrt(5.0))
    angles = np.arange(spokes, dtype=np.float64) * golden
    radius = np.linspace(-0.5, 0.5, readout, endpoint=False, dtype=np.float64)
    k0 = np.cos(angles)[:, None] * radius[None, :]
    k1 = np.sin(angles)[:, None] * radius[None, :]
    return np.stack((k0, k1), axis=-1).reshape(-1, 2).astype(np.float32)


def vd_spiral(interleaves: int, samples: int, exponent: float = 1.5, turns: float | None = None) -> np.ndarray:
    """[interleaves*samples, 2] float32 variable-density spiral (cycles/pixel)."""
    if turns is None:
        turns = max(4.0, samples / 256.0)
    t = (np.arange(samples, dtype=np.float64) + 0.5) / samples
    radius = 0.499 * t ** exponent
    out = []
    for i in range(interleaves):
        theta = 2.0 * math.pi * (turns * t + i / interleaves)
        out.append(np.stack((radius * np.cos(theta), radius * np.sin(theta)), axis=-1))
    return np.concatenate(out, axis=0).astype(np.float32)


def ramp_density(trajectory: np.ndarray, readout: int | None = None) -> np.ndarray:
    """[M] float32 ramp density compensation, max 1: |k| for [M, 2] trajectories and |k|^2
    for [M, 3] (3D radial), with |k| floored at half a readout step."""
    traj = np.asarray(trajectory, dtype=np.float64)
    dims = traj.shape[-1] if traj.ndim == 2 and traj.shape[-1] in (2, 3) else 2
    k = np.linalg.norm(traj.reshape(-1, dims), axis=1)
    floor = 1.0 / (readout if readout else 512)
    w = np.maximum(k, 0.5 * floor) ** (dims - 1)
    return (w / w.max()).astype(np.float32)


def add_noise(samples: np.ndarray, seed: int, level: float = 1e-3) -> np.ndarray:
    """complex Gaussian noise at ``level`` x rms of ``samples``."""
    rng = np.random.default_rng(seed + 104729)
    rms = math.sqrt(float(np.mean(np.abs(samples.astype(np.complex128)) ** 2)))
    noise = rng.standard_normal(samples.shape) + 1j * rng.standard_normal(samples.shape)
    return (samples + level * rms / math.sqrt(2.0) * noise).astype(np.complex64)


def uneven_batch(count: int = 48, seed: int = BASE_SEED) -> list[dict]:
    """Seeded uneven batch: image size N from {128, 192, 256, 320} (grid 2N), coils from
    {4, 8, 12, 16}; even cases golden-angle radial (64-384 spokes x 2N samples), odd cases
    variable-density spirals (8-32 interleaves x 2048-4096 samples, density exponent 1.5).
    Case i uses seed + i for its phantom, coils and noise."""
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(count):
        n = int(rng.choice([128, 192, 256, 320]))
        c = int(rng.choice([4, 8, 12, 16]))
        if i % 2 == 0:
            spokes = int(rng.integers(64, 385))
            traj = golden_radial(spokes, 2 * n)
            kind = f"radial {spokes}x{2 * n}"
        else:
            inter = int(rng.integers(8, 33))
            samples = int(rng.integers(2048, 4097))
            traj = vd_spiral(inter, samples, 1.5)
            kind = f"spiral {inter}x{samples}"
        cases.append({"n": n, "g": 2 * n, "c": c, "trajectory": traj, "kind": kind, "seed": seed + i})
    return cases


# ---- volumes (3D kooshball) -----------------------------------------------------------------
def _grid3(n: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    coords = (np.arange(n, dtype=np.float64) - n // 2) / n
    return np.meshgrid(coords, coords, coords, indexing="ij")


def ellipsoid_phantom(n: int, seed: int, ellipsoids: int = 12) -> np.ndarray:
    """[N, N, N] complex64 phantom: random ellipsoids (magnitudes U(0.1, 1), random
    orientation) times a smooth linear-ramp phase."""
    rng = np.random.default_rng(seed)
    z, y, x = _grid3(n)
    vol = np.zeros((n, n, n), dtype=np.float64)
    for _ in range(ellipsoids):
        centre = rng.uniform(-0.25, 0.25, size=3)
        axes = rng.uniform(0.05, 0.3, size=3)
        # random rotation from a QR of a Gaussian matrix (det fixed to +1)
        q, r = np.linalg.qr(rng.standard_normal((3, 3)))
        q = q * np.sign(np.diag(r))[None, :]
        if np.linalg.det(q) < 0:
            q[:, 0] = -q[:, 0]
        mag = rng.uniform(0.1, 1.0)
        d = np.stack((z - centre[0], y - centre[1], x - centre[2]), axis=-1)
        local = d @ q
        inside = ((local / axes) ** 2).sum(axis=-1) <= 1.0
        vol += mag * inside
    slope = rng.uniform(-1.0, 1.0, size=3)
    phase = np.exp(1j * math.pi * (slope[0] * z + slope[1] * y + slope[2] * x))
    return (vol * phase).astype(np.complex64)


def coil_maps3(n: int, coils: int, seed: int) -> np.ndarray:
    """[C, N, N, N] complex64 Gaussian-blob sensitivities with centres spread on a sphere of
    radius 0.7 FOV (Fibonacci lattice), sigma 0.4 FOV, random linear phase, RSS = 1."""
    rng = np.random.default_rng(seed + 7919)
    z, y, x = _grid3(n)
    maps = np.zeros((coils, n, n, n), dtype=np.complex128)
    golden = math.pi * (3.0 - math.sqrt(5.0))
    for c in range(coils):
        cz = 1.0 - 2.0 * (c + 0.5) / coils
        ring = math.sqrt(max(0.0, 1.0 - cz * cz))
        centre = 0.7 * np.array([cz, ring * math.sin(golden * c), ring * math.cos(golden * c)])
        blob = np.exp(-((z - centre[0]) ** 2 + (y - centre[1]) ** 2 + (x - centre[2]) ** 2) / (2.0 * 0.4 ** 2))
        slope = rng.uniform(-1.0, 1.0, size=3)
        maps[c] = blob * np.exp(1j * math.pi * (slope[0] * z + slope[1] * y + slope[2] * x))
    rss = np.sqrt(np.sum(np.abs(maps) ** 2, axis=0))
    return (maps / rss).astype(np.complex64)


# 3D golden means for radial sampling (Chan et al., MRM 2009): phi2 is the real root of
# x^3 + x - 1 = 0 and phi1 = phi2^2
GOLDEN_MEANS_3D = (0.465571231876768, 0.682327803828019)


def kooshball(spokes: int, readout: int) -> np.ndarray:
    """[spokes*readout, 3] float32 golden-means 3D radial trajectory (cycles/pixel): spoke m
    has direction cos(polar) = 2 frac(m phi1) - 1, azimuth 2 pi frac(m phi2), and samples
    linspace(-0.5, 0.5, readout, endpoint=False) along it."""
    m = np.arange(spokes, dtype=np.float64)
    kz = 2.0 * np.mod(m * GOLDEN_MEANS_3D[0], 1.0) - 1.0
    az = 2.0 * math.pi * np.mod(m * GOLDEN_MEANS_3D[1], 1.0)
    ring = np.sqrt(np.maximum(0.0, 1.0 - kz * kz))
    direction = np.stack((kz, ring * np.sin(az), ring * np.cos(az)), axis=-1)  # [spokes, 3]
    radius = np.linspace(-0.5, 0.5, readout, endpoint=False, dtype=np.float64)
    traj = direction[:, None, :] * radius[None, :, None]
    return traj.reshape(-1, 3).astype(np.float32)
