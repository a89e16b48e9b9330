"""Seeded GPU test cases and oracle helpers (tests only)."""
from __future__ import annotations

import functools
import math

import numpy as np

from oracle import nudft as onudft
from oracle import operator as oop
from trajsparsenufft_b200 import synth

SEED = synth.BASE_SEED


@functools.lru_cache(maxsize=None)
def case(name: str):
    """(trajectory, image, smaps, N, G, C, J, readout) of a named configuration."""
    if name == "small":
        n, g, c, spokes, readout = 64, 128, 4, 48, 128
    elif name == "cfg0":          # 128^2, 4 coils, 96 x 256 golden-angle radial
        n, g, c, spokes, readout = 128, 256, 4, 96, 256
    elif name == "headline":      # 256^2, 8 coils, 256 x 512 golden-angle radial
        n, g, c, spokes, readout = 256, 512, 8, 256, 512
    elif name == "grad4":         # one case of the differentiable config: 4x-undersampled radial
        n, g, c, spokes, readout = 256, 512, 8, 128, 512
    elif name == "c16":
        n, g, c, spokes, readout = 128, 256, 16, 64, 256
    elif name == "n192":          # grid 384 = 3 x 128: radix-3 FFT step
        n, g, c, spokes, readout = 192, 384, 4, 24, 384
    elif name == "n320":          # grid 640 = 5 x 128: radix-5 FFT step, 12 coils
        n, g, c, spokes, readout = 320, 640, 12, 16, 640
    else:
        raise KeyError(name)
    traj = synth.golden_radial(spokes, readout)
    x = synth.ellipse_phantom(n, SEED)
    s = synth.coil_maps(n, c, SEED)
    return traj, x, s, n, g, c, 6, readout


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def oracle_cg(forward, adjoint, y, density, iters, lam):
    w = None if density is None else np.asarray(density, dtype=np.float64)
    adj = adjoint if w is None else (lambda v: adjoint(w[None] * v))
    return oop.cg_sense(forward, adj, y, iters, lam)


@functools.lru_cache(maxsize=None)
def measurement(name: str):
    """FP64 direct NUDFT k-space + 1e-3 rms complex noise (the config 0 recipe; the headline's
    131072 x 65536 x 8 NUDFT takes a few seconds as chunked GEMMs)."""
    traj, x, s, n, *_ = case(name)
    y = onudft.Nudft(traj, n).forward(x, s)
    return synth.add_noise(y, SEED)


def torch_inputs(name: str, dev="cuda"):
    import torch
    traj, x, s, *_ = case(name)
    y = measurement(name)
    return (torch.from_numpy(np.ascontiguousarray(x)).to(dev), torch.from_numpy(np.ascontiguousarray(s)).to(dev),
            torch.from_numpy(np.ascontiguousarray(y)).to(dev))


@functools.lru_cache(maxsize=None)
def volume_case(name: str):
    """(trajectory [M,3], volume, smaps, N, G, C, J) of a named 3D kooshball configuration."""
    if name == "vol64":           # 64^3 on a 128^3 grid, 4 coils, 512 x 128 golden-means kooshball
        n, g, c, spokes, readout = 64, 128, 4, 512, 128
    elif name == "vol64c8":       # 8 coils, sparser
        n, g, c, spokes, readout = 64, 128, 8, 256, 128
    else:
        raise KeyError(name)
    traj = synth.kooshball(spokes, readout)
    x = synth.ellipsoid_phantom(n, SEED)
    s = synth.coil_maps3(n, c, SEED)
    return traj, x, s, n, g, c, 4


@functools.lru_cache(maxsize=None)
def volume_measurement(name: str):
    """k-space of a volume case from the FP64 KB operator with J = 6 (within ~1e-5 of the direct
    NUDFT; the NUDFT itself is checked on a subsample) plus 1e-3 rms complex noise."""
    traj, x, s, n, g, c, _ = volume_case(name)
    y = oop.KbSenseOperator3(traj, n, g, 6, workers=8).forward(x, s)
    return synth.add_noise(y, SEED)
