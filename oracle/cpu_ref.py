"""FP32 CPU CG-SENSE: the reference's own CPU code path, restated (timed CPU baseline).

TEST INFRASTRUCTURE / BASELINE: see oracle/__init__.py.  Used by bench.py's
``cpu_baseline`` leg and ``--impl reference`` arm only.

Restates experiments/production/reference_sparse_solver.py with
``make_component_operator(..., "fp32", "fp32", device=cpu, "csr")`` (:131-197) and
``cg_sense`` (:200-332): separate real/imag FP32 CSR matrices and their transposes,
panel products summed as in ``sum_sparse_products`` (:121-128), pad -> FFT -> scale
(the torchkbnufft ``fft_and_scale`` role) and its inverse, complex64 vectors.
The sparse products run row-blocked on a thread pool (scipy releases the GIL) and
the FFTs use scipy.fft workers, so the baseline uses every host core it is given.
"""

from __future__ import annotations

import math
import os
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.fft
import scipy.sparse as sp

from . import kb


class CpuSenseFp32:
    def __init__(self, trajectory, im_size: int, grid_size: int, width: int, smaps, threads: int | None = None):
        self.n, self.g = im_size, grid_size
        self.threads = threads or os.cpu_count() or 1
        self.pool = ThreadPoolExecutor(self.threads)
        row_ptr, cols, re, im = kb.interpolation_csr(trajectory, im_size, grid_size, width)
        m = len(row_ptr) - 1
        shape = (m, grid_size * grid_size)
        g_re = sp.csr_matrix((re.astype(np.float32), cols, row_ptr), shape=shape)
        g_im = sp.csr_matrix((im.astype(np.float32), cols, row_ptr), shape=shape)
        self.m = m
        self.fwd = (self._blocks(g_re), self._blocks(g_im))
        self.adj = (self._blocks(g_re.T.tocsr()), self._blocks(g_im.T.tocsr()))
        self.scaling = kb.deapodization(im_size, grid_size, width).astype(np.float32)
        self.smaps = np.asarray(smaps, dtype=np.complex64)
        self.c = self.smaps.shape[0]

    def _blocks(self, mat):
        rows = mat.shape[0]
        step = max(1, math.ceil(rows / self.threads))
        return [mat[i:i + step] for i in range(0, rows, step)]

    def _mm(self, blocks, panel):
        return np.concatenate(list(self.pool.map(lambda b: b @ panel, blocks)), axis=0)

    def forward(self, image):
        coil = (image[None] * self.smaps) * self.scaling[None]
        grid = np.zeros((self.c, self.g, self.g), dtype=np.complex64)
        grid[:, : self.n, : self.n] = coil
        z = scipy.fft.fft2(grid, workers=self.threads)
        panel = z.reshape(self.c, -1).T
        pr, pi = np.ascontiguousarray(panel.real), np.ascontiguousarray(panel.imag)
        gr, gi = self.fwd
        out_re = self._mm(gr, pr) - self._mm(gi, pi)
        out_im = self._mm(gr, pi) + self._mm(gi, pr)
        return (out_re + 1j * out_im).astype(np.complex64).T

    def adjoint(self, data):
        panel = np.asarray(data).T
        pr, pi = np.ascontiguousarray(panel.real), np.ascontiguousarray(panel.imag)
        tr, ti = self.adj
        grid_re = self._mm(tr, pr) + self._mm(ti, pi)
        grid_im = self._mm(tr, pi) - self._mm(ti, pr)
        grid = (grid_re + 1j * grid_im).astype(np.complex64).T.reshape(self.c, self.g, self.g)
        img = scipy.fft.ifft2(grid, workers=self.threads) * np.float32(self.g * self.g)
        coil = img[:, : self.n, : self.n] * self.scaling[None]
        return np.sum(np.conj(self.smaps) * coil, axis=0).astype(np.complex64)

    def cg_sense(self, data, iterations: int, lam: float, sample_iterations: int | None = None):
        """FP32 CG of reference_sparse_solver.cg_sense; returns (x, residuals, seconds of
        the right-hand side, seconds per iteration)."""
        t0 = time.perf_counter()
        b = self.adjoint(data)
        t_rhs = time.perf_counter() - t0
        x = np.zeros_like(b)
        r = b.copy()
        p = r.copy()
        rs_old = np.float32(np.vdot(r, r).real)
        res = [float(np.sqrt(max(rs_old, 0.0)))]
        run = iterations if sample_iterations is None else min(iterations, sample_iterations)
        t1 = time.perf_counter()
        for _ in range(run):
            ap = self.adjoint(self.forward(p)) + np.float32(lam) * p
            den = np.float32(np.vdot(p, ap).real)
            if not np.isfinite(den) or den <= 0:
                break
            alpha = rs_old / max(den, np.float32(1e-30))
            x = x + alpha * p
            r = r - alpha * ap
            rs_new = np.float32(np.vdot(r, r).real)
            res.append(float(np.sqrt(max(rs_new, 0.0))))
            p = r + (rs_new / max(rs_old, np.float32(1e-30))) * p
            rs_old = rs_new
        t_iter = (time.perf_counter() - t1) / max(run, 1)
        return x, res, t_rhs, t_iter
