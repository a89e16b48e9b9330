"""FP64 direct non-uniform DFT with SENSE coil maps (accuracy oracle).

TEST INFRASTRUCTURE: see oracle/__init__.py.

Forward:  y_c[m] = sum_{i0,i1} S_c[i0,i1] x[i0,i1] exp(-i (w0_m (i0-c) + w1_m (i1-c)))
Adjoint:  x[i0,i1] = sum_c conj(S_c[i0,i1]) sum_m y_c[m] exp(+i (...))
with w = 2*pi*k (k in cycles/pixel, the reference's trajectory contract,
experiments/data_prep/generate_trajectories.py:43-49) and c = N//2.

The 2D sum is separable, so both directions are evaluated exactly as dense
complex128 GEMMs over sample chunks (cost M*N^2 per coil, no approximation);
Nudft3 is the same for volumes (cost M*N^3 per coil).
The reference has no direct NUDFT; it measures against torchkbnufft tables.
"""

from __future__ import annotations

import numpy as np


class Nudft:
    def __init__(self, trajectory: np.ndarray, im_size: int, chunk: int = 16384):
        traj = np.asarray(trajectory, dtype=np.float64).reshape(-1, 2)
        self.n = im_size
        self.m = traj.shape[0]
        self.chunk = chunk
        t = np.arange(im_size, dtype=np.float64) - im_size // 2
        self._w = 2.0 * np.pi * traj
        self._t = t

    def _basis(self, lo: int, hi: int):
        w = self._w[lo:hi]
        e0 = np.exp(-1j * np.outer(w[:, 0], self._t))
        e1 = np.exp(-1j * np.outer(w[:, 1], self._t))
        return e0, e1

    def forward(self, image: np.ndarray, smaps: np.ndarray | None = None) -> np.ndarray:
        """image [N,N] (or coil images [C,N,N] when smaps is None) -> samples [C,M]."""
        x = np.asarray(image, dtype=np.complex128)
        coil_images = x[None] * np.asarray(smaps, dtype=np.complex128) if smaps is not None else x
        c = coil_images.shape[0]
        n = self.n
        # stacked right-hand side: [N(i1), C*N(i0)]
        rhs = coil_images.transpose(2, 0, 1).reshape(n, c * n)
        out = np.empty((c, self.m), dtype=np.complex128)
        for lo in range(0, self.m, self.chunk):
            hi = min(self.m, lo + self.chunk)
            e0, e1 = self._basis(lo, hi)
            t = (e1 @ rhs).reshape(hi - lo, c, n)          # [m, c, i0]
            out[:, lo:hi] = np.einsum("mci,mi->cm", t, e0)
        return out

    def adjoint(self, samples: np.ndarray, smaps: np.ndarray | None = None) -> np.ndarray:
        """samples [C,M] -> image [N,N] (coil-combined) or coil images [C,N,N]."""
        y = np.asarray(samples, dtype=np.complex128)
        c = y.shape[0]
        n = self.n
        acc = np.zeros((c, n, n), dtype=np.complex128)
        for lo in range(0, self.m, self.chunk):
            hi = min(self.m, lo + self.chunk)
            e0, e1 = self._basis(lo, hi)
            e0c = np.conj(e0)
            e1c = np.conj(e1)
            for coil in range(c):
                acc[coil] += e0c.T @ (y[coil, lo:hi, None] * e1c)
        if smaps is None:
            return acc
        return np.sum(np.conj(np.asarray(smaps, dtype=np.complex128)) * acc, axis=0)


class Nudft3:
    """FP64 direct 3D NUDFT with SENSE maps:
    y_c[m] = sum_i S_c[i] x[i] exp(-i sum_d w_d,m (i_d - c)), w = 2 pi k, c = N//2.
    Separable: the i2 sum is a GEMM over a chunk of samples, the i1 and i0 sums are
    per-sample contractions (cost C*N^3*M, exact)."""

    def __init__(self, trajectory: np.ndarray, im_size: int):
        traj = np.asarray(trajectory, dtype=np.float64).reshape(-1, 3)
        self.n = im_size
        self.m = traj.shape[0]
        self._w = 2.0 * np.pi * traj
        self._t = np.arange(im_size, dtype=np.float64) - im_size // 2

    def _chunk(self, c: int) -> int:
        return max(1, int(2 ** 27 // (16 * c * self.n * self.n)))

    def _basis(self, lo: int, hi: int, d: int):
        return np.exp(-1j * np.outer(self._w[lo:hi, d], self._t))   # [s, N]

    def forward(self, image: np.ndarray, smaps: np.ndarray | None = None) -> np.ndarray:
        """image [N,N,N] (or coil volumes [C,N,N,N] when smaps is None) -> samples [C,M]."""
        x = np.asarray(image, dtype=np.complex128)
        v = x[None] * np.asarray(smaps, dtype=np.complex128) if smaps is not None else x
        c, n = v.shape[0], self.n
        flat = v.reshape(c * n * n, n)
        out = np.empty((c, self.m), dtype=np.complex128)
        step = self._chunk(c)
        for lo in range(0, self.m, step):
            hi = min(self.m, lo + step)
            e0, e1, e2 = (self._basis(lo, hi, d) for d in range(3))
            t1 = (flat @ e2.T).reshape(c, n, n, hi - lo)            # [c, i0, i1, s]
            t2 = np.einsum("cabs,sb->cas", t1, e1)                  # [c, i0, s]
            out[:, lo:hi] = np.einsum("cas,sa->cs", t2, e0)
        return out

    def adjoint(self, samples: np.ndarray, smaps: np.ndarray | None = None) -> np.ndarray:
        """samples [C,M] -> volume [N,N,N] (coil-combined) or coil volumes [C,N,N,N]."""
        y = np.asarray(samples, dtype=np.complex128)
        c, n = y.shape[0], self.n
        acc = np.zeros((c * n * n, n), dtype=np.complex128)
        step = self._chunk(c)
        for lo in range(0, self.m, step):
            hi = min(self.m, lo + step)
            e0, e1, e2 = (np.conj(self._basis(lo, hi, d)) for d in range(3))
            a1 = y[:, None, lo:hi] * e0.T[None]                         # [c, i0, s]
            a2 = a1[:, :, None, :] * e1.T[None, None]                   # [c, i0, i1, s]
            acc += a2.reshape(c * n * n, hi - lo) @ e2                  # [c*i0*i1, i2]
        vol = acc.reshape(c, n, n, n)
        if smaps is None:
            return vol
        return np.sum(np.conj(np.asarray(smaps, dtype=np.complex128)) * vol, axis=0)
