"""Kaiser-Bessel interpolation coefficients and deapodization in FP64 (oracle).

TEST INFRASTRUCTURE: see oracle/__init__.py.

The reference obtains its production coefficient matrix from
``torchkbnufft.calc_tensor_spmatrix`` (src/export_torchkbnufft_gpu_case.py:537-567)
and its deapodization table from ``KbNufft.scaling_coef``
(experiments/data_prep/export_real_runtime_inputs.py:97-101).  torchkbnufft
1.5.2 is not vendored, so this module restates the published gridding NUFFT
(Jackson et al. 1991; Beatty et al. 2005) with the reference's own kernel:

* kernel  phi(d) = I0(beta*sqrt(1-(2d/J)^2)) / I0(beta), |d| < J/2, else 0
          (same expression as src/nufft_layout_oracle.py:152-156)
* beta    = pi*sqrt((J/alpha*(alpha-0.5))^2 - 0.8)   (src/nufft_layout_oracle.py:168-169)
* support J points per axis starting at floor(u - J/2) + 1, u = k*G in grid units
* phase   exp(2*pi*i*q*c/G) per grid index q with c = N//2 — this carries the
          image placement at [0, N) of the padded grid (the reference's FFT
          endpoint convention, nufft_custom_fft_forward_bench.cu:1600-1844)
* deapod  1 / (Phi(t0/G) * Phi(t1/G)), t = i - N//2, with Phi the continuous
          Fourier transform of phi: J*sinh(z)/z / I0(beta), z^2 = beta^2-(pi*J*xi)^2

With these definitions  sum_i x[i] exp(-i w.(i-c))  ~=  sum_q C[m,q] FFT_G(pad(x*deapod))[q]
for a trajectory w = 2*pi*k, k in cycles/pixel in [-0.5, 0.5).
"""

from __future__ import annotations

import math

import numpy as np


def beatty_beta(width: int, oversampling: float = 2.0) -> float:
    term = (width / oversampling * (oversampling - 0.5)) ** 2 - 0.8
    return math.pi * math.sqrt(max(term, 0.01))


def kb_weight(distance: np.ndarray, width: int, beta: float) -> np.ndarray:
    scaled = 2.0 * np.asarray(distance, dtype=np.float64) / width
    inside = np.abs(scaled) < 1.0
    arg = beta * np.sqrt(np.maximum(0.0, 1.0 - scaled * scaled))
    return np.where(inside, np.i0(arg) / np.i0(beta), 0.0)


def kb_fourier(xi: np.ndarray, width: int, beta: float) -> np.ndarray:
    """Continuous Fourier transform of kb_weight at frequency xi (cycles/grid unit)."""
    xi = np.asarray(xi, dtype=np.float64)
    z2 = beta * beta - (math.pi * width * xi) ** 2
    z = np.sqrt(np.abs(z2))
    with np.errstate(divide="ignore", invalid="ignore"):
        pos = np.where(z > 0, np.sinh(z) / np.where(z > 0, z, 1.0), 1.0)
        neg = np.where(z > 0, np.sin(z) / np.where(z > 0, z, 1.0), 1.0)
    return width * np.where(z2 >= 0, pos, neg) / np.i0(beta)


def deapodization(im_size: int, grid_size: int, width: int, beta: float | None = None) -> np.ndarray:
    """[N, N] real deapodization table (the runtime ``scaling.f32.bin`` role)."""
    if beta is None:
        beta = beatty_beta(width, grid_size / im_size)
    t = np.arange(im_size, dtype=np.float64) - im_size // 2
    inv = 1.0 / kb_fourier(t / grid_size, width, beta)
    return np.outer(inv, inv)


def exact_phase(k: np.ndarray, grid_size: int) -> tuple[np.ndarray, np.ndarray]:
    """cos/sin of 2*pi*k/G for integer k, exact at multiples of G/4."""
    k = np.mod(np.asarray(k, dtype=np.int64), grid_size)
    quarter = (4 * k) % grid_size == 0
    q = (4 * k) // grid_size
    cos_exact = np.choose(np.where(quarter, q, 0) % 4, [1.0, 0.0, -1.0, 0.0])
    sin_exact = np.choose(np.where(quarter, q, 0) % 4, [0.0, 1.0, 0.0, -1.0])
    angle = 2.0 * math.pi * k / grid_size
    return (np.where(quarter, cos_exact, np.cos(angle)),
            np.where(quarter, sin_exact, np.sin(angle)))


def interpolation_csr(trajectory: np.ndarray, im_size: int, grid_size: int, width: int,
                      beta: float | None = None):
    """Complex KB interpolation matrix as CSR (row_ptr, cols, re, im), FP64.

    Rows are samples in trajectory order; within a row the columns (grid cell
    q0*G + q1, axis 0 of the trajectory pairing with axis 0 of the image) are
    sorted ascending and exact-zero weights are dropped, as
    src/nufft_layout_oracle.py:185-194 does for its real matrix.
    """
    if beta is None:
        beta = beatty_beta(width, grid_size / im_size)
    traj = np.asarray(trajectory, dtype=np.float64).reshape(-1, 2)
    m = traj.shape[0]
    u = traj * grid_size
    start = np.floor(u - width / 2.0).astype(np.int64) + 1
    q = start[:, :, None] + np.arange(width, dtype=np.int64)[None, None, :]
    w = kb_weight(u[:, :, None] - q, width, beta)
    c = im_size // 2
    w2 = w[:, 0, :, None] * w[:, 1, None, :]
    kphase = q[:, 0, :, None] * c + q[:, 1, None, :] * c
    cos_p, sin_p = exact_phase(kphase, grid_size)
    cols = (np.mod(q[:, 0, :, None], grid_size) * grid_size
            + np.mod(q[:, 1, None, :], grid_size)).reshape(m, -1)
    w2 = w2.reshape(m, -1)
    re = (w2 * cos_p.reshape(m, -1))
    im = (w2 * sin_p.reshape(m, -1))
    order = np.argsort(cols, axis=1, kind="stable")
    cols = np.take_along_axis(cols, order, axis=1)
    w2 = np.take_along_axis(w2, order, axis=1)
    re = np.take_along_axis(re, order, axis=1)
    im = np.take_along_axis(im, order, axis=1)
    keep = w2 != 0.0
    counts = keep.sum(axis=1)
    row_ptr = np.zeros(m + 1, dtype=np.int64)
    row_ptr[1:] = np.cumsum(counts)
    return row_ptr, cols[keep].astype(np.int64), re[keep], im[keep]


def to_scipy(row_ptr, cols, re, im, n_cols):
    import scipy.sparse as sp
    vals = re + 1j * im
    return sp.csr_matrix((vals, cols, row_ptr), shape=(len(row_ptr) - 1, n_cols))


def weights_csr3(trajectory: np.ndarray, im_size: int, grid_size: int, width: int,
                 beta: float | None = None):
    """3D real KB weights as CSR (row_ptr, cols, w), FP64, for the centred-image layout.

    The image sits centred on the grid (grid position n holds image index
    (n + N//2) mod G), so the phase exp(2*pi*i*q.c/G) of the corner layout is
    not needed and the coefficients are the real tensor-product weights
    w = (phi(u0-q0) * phi(u1-q1)) * phi(u2-q2).  Rows are samples in
    trajectory order; columns are cells (q0*G + q1)*G + q2 with q_d wrapped
    mod G, sorted ascending; exact zeros are dropped.  The 2D rules of
    interpolation_csr extended by one axis (the reference itself is 2D only).
    """
    if beta is None:
        beta = beatty_beta(width, grid_size / im_size)
    traj = np.asarray(trajectory, dtype=np.float64).reshape(-1, 3)
    m = traj.shape[0]
    u = traj * grid_size
    start = np.floor(u - width / 2.0).astype(np.int64) + 1
    q = start[:, :, None] + np.arange(width, dtype=np.int64)[None, None, :]   # [m, 3, J]
    w = kb_weight(u[:, :, None] - q, width, beta)
    wq = np.mod(q, grid_size)
    w3 = (w[:, 0, :, None, None] * w[:, 1, None, :, None]) * w[:, 2, None, None, :]
    cols = ((wq[:, 0, :, None, None] * grid_size + wq[:, 1, None, :, None]) * grid_size
            + wq[:, 2, None, None, :])
    w3 = w3.reshape(m, -1)
    cols = cols.reshape(m, -1)
    order = np.argsort(cols, axis=1, kind="stable")
    cols = np.take_along_axis(cols, order, axis=1)
    w3 = np.take_along_axis(w3, order, axis=1)
    keep = w3 != 0.0
    row_ptr = np.zeros(m + 1, dtype=np.int64)
    row_ptr[1:] = np.cumsum(keep.sum(axis=1))
    return row_ptr, cols[keep].astype(np.int64), w3[keep]


def deapodization3(im_size: int, grid_size: int, width: int, beta: float | None = None) -> np.ndarray:
    """[N, N, N] real deapodization (inv[a] * inv[b]) * inv[c]."""
    if beta is None:
        beta = beatty_beta(width, grid_size / im_size)
    t = np.arange(im_size, dtype=np.float64) - im_size // 2
    inv = 1.0 / kb_fourier(t / grid_size, width, beta)
    return (inv[:, None, None] * inv[None, :, None]) * inv[None, None, :]
