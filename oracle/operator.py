"""KB SENSE NUFFT operators and the CG-SENSE recursion (oracle).

TEST INFRASTRUCTURE: see oracle/__init__.py.

``KbSenseOperator`` restates ``make_component_operator``
(experiments/production/reference_sparse_solver.py:131-197): SENSE multiply,
deapodize and zero-pad at [0, N) of the G x G grid, unnormalized forward FFT
(the torchkbnufft ``fft_and_scale`` role), then the complex component sparse
products (real/imag matrices, each optionally FP16, the dense panel FP64, FP32,
FP16 or the FP16 high + FP16 residual split of ``dense_components`` :66-76).
The adjoint is the exact conjugate transpose: conjugated component products,
unnormalized inverse FFT, crop, deapodize, coil combine with conj(S).

``KbSenseOperator3`` is the same operator for volumes (real weights, centred image).

``cg_sense`` restates the CG recursion with its status dictionary
(reference_sparse_solver.py:200-332, without the reliable-update options);
``cg_sense_scheduled`` adds its scheduled reference steps.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.fft
import scipy.sparse as sp

from . import kb

PANEL_MODES = ("fp64", "fp32", "fp16", "split2")
MATRIX_MODES = ("fp64", "fp32", "fp16", "fp16x2")


def _quantize_matrix(values: np.ndarray, mode: str) -> np.ndarray:
    if mode == "fp64":
        return values
    if mode == "fp32":
        return values.astype(np.float32).astype(np.float64)
    if mode == "fp16":
        return values.astype(np.float16).astype(np.float64)
    if mode == "fp16x2":  # FP16 high part + FP16 residual (the FP32-class reference-step views)
        hi = values.astype(np.float16).astype(np.float64)
        return hi + (values - hi).astype(np.float16).astype(np.float64)
    raise ValueError(mode)


def pow2_scale(values: np.ndarray, target: float = 64.0) -> float:
    """Power-of-two factor that brings rms(values) near ``target``.

    Scaling by a power of two commutes with FP16 rounding away from the
    subnormal and overflow ranges, so the split below matches an unscaled
    split while staying inside FP16 range.
    """
    rms = math.sqrt(float(np.mean(np.abs(values) ** 2))) if values.size else 0.0
    if not math.isfinite(rms) or rms == 0.0:
        return 1.0
    return 2.0 ** round(math.log2(target / rms))


def dense_components(panel: np.ndarray, mode: str) -> np.ndarray:
    """Effective panel after the reference's dense_components (real arrays)."""
    if mode == "fp64":
        return panel
    v32 = panel.astype(np.float32)
    if mode == "fp32":
        return v32.astype(np.float64)
    scale = pow2_scale(v32.astype(np.float64))
    vs = (v32.astype(np.float64) * scale).astype(np.float32)
    hi = vs.astype(np.float16).astype(np.float32)
    if mode == "fp16":
        return hi.astype(np.float64) / scale
    res = (vs - hi).astype(np.float16).astype(np.float32)
    return (hi.astype(np.float64) + res.astype(np.float64)) / scale


class KbSenseOperator:
    """Forward / adjoint SENSE NUFFT with KB interpolation (complex components)."""

    def __init__(self, trajectory, im_size: int, grid_size: int, width: int,
                 matrix_mode: str = "fp64", panel_mode: str = "fp64",
                 csr=None, scaling: np.ndarray | None = None, workers: int = 1):
        self.n = im_size
        self.g = grid_size
        self.workers = workers
        self.panel_mode = panel_mode
        if csr is None:
            csr = kb.interpolation_csr(trajectory, im_size, grid_size, width)
        row_ptr, cols, re, im = csr
        re = _quantize_matrix(re, matrix_mode)
        im = _quantize_matrix(im, matrix_mode)
        m = len(row_ptr) - 1
        shape = (m, grid_size * grid_size)
        self.m = m
        self.g_re = sp.csr_matrix((re, cols, row_ptr), shape=shape)
        self.g_im = sp.csr_matrix((im, cols, row_ptr), shape=shape)
        self.gt_re = self.g_re.T.tocsr()
        self.gt_im = self.g_im.T.tocsr()
        if scaling is None:
            scaling = kb.deapodization(im_size, grid_size, width)
        self.scaling = np.asarray(scaling, dtype=np.float64)

    def grid_panel(self, image, smaps) -> np.ndarray:
        """[G*G, C] complex panel = FFT(pad(x * S_c * scaling))."""
        coil = np.asarray(image, dtype=np.complex128)[None] * np.asarray(smaps, dtype=np.complex128)
        coil = coil * self.scaling[None]
        c = coil.shape[0]
        grid = np.zeros((c, self.g, self.g), dtype=np.complex128)
        grid[:, : self.n, : self.n] = coil
        z = scipy.fft.fft2(grid, workers=self.workers)
        return z.reshape(c, -1).T

    def interp(self, panel: np.ndarray) -> np.ndarray:
        pr = dense_components(panel.real, self.panel_mode)
        pi = dense_components(panel.imag, self.panel_mode)
        out_re = self.g_re @ pr - self.g_im @ pi
        out_im = self.g_re @ pi + self.g_im @ pr
        return (out_re + 1j * out_im).T

    def interp_adjoint(self, samples: np.ndarray) -> np.ndarray:
        panel = np.asarray(samples).T
        pr = dense_components(panel.real, self.panel_mode)
        pi = dense_components(panel.imag, self.panel_mode)
        grid_re = self.gt_re @ pr + self.gt_im @ pi
        grid_im = self.gt_re @ pi - self.gt_im @ pr
        return (grid_re + 1j * grid_im).T

    def forward(self, image, smaps) -> np.ndarray:
        return self.interp(self.grid_panel(image, smaps))

    def adjoint_coils(self, samples) -> np.ndarray:
        grid = self.interp_adjoint(samples)
        c = grid.shape[0]
        grid = grid.reshape(c, self.g, self.g)
        img = scipy.fft.ifft2(grid, workers=self.workers) * float(self.g * self.g)
        return img[:, : self.n, : self.n] * self.scaling[None]

    def adjoint(self, samples, smaps) -> np.ndarray:
        coil = self.adjoint_coils(samples)
        return np.sum(np.conj(np.asarray(smaps, dtype=np.complex128)) * coil, axis=0)


class KbSenseOperator3:
    """Volume SENSE NUFFT with real KB weights on the centred layout (FP64 by default).

    Forward: x * S_c * deapodization placed centred on the G^3 grid (image index i at
    grid position (i - N//2) mod G on every axis), unnormalized 3D FFT, then the real
    weight matrix of kb.weights_csr3 (cells (q0*G + q1)*G + q2).  Adjoint: the exact
    conjugate transpose.  matrix_mode / panel_mode emulate the FP16 weights and the
    FP16 high + residual panels as KbSenseOperator does for images.
    """

    def __init__(self, trajectory, im_size: int, grid_size: int, width: int,
                 matrix_mode: str = "fp64", panel_mode: str = "fp64", workers: int = 1):
        self.n = im_size
        self.g = grid_size
        self.workers = workers
        self.panel_mode = panel_mode
        row_ptr, cols, w = kb.weights_csr3(trajectory, im_size, grid_size, width)
        w = _quantize_matrix(w, matrix_mode)
        self.m = len(row_ptr) - 1
        self.w = sp.csr_matrix((w, cols, row_ptr), shape=(self.m, grid_size ** 3))
        self.wt = self.w.T.tocsr()
        self.scaling = kb.deapodization3(im_size, grid_size, width)
        self._pos = (np.arange(im_size) - im_size // 2) % grid_size

    def grid_panel(self, image, smaps) -> np.ndarray:
        """[G^3, C] complex panel = FFT3(centred pad(x * S_c * scaling))."""
        coil = np.asarray(image, dtype=np.complex128)[None] * np.asarray(smaps, dtype=np.complex128)
        return self.grid_panel_coils(coil)

    def grid_panel_coils(self, coil) -> np.ndarray:
        coil = np.asarray(coil, dtype=np.complex128) * self.scaling[None]
        c, g, pos = coil.shape[0], self.g, self._pos
        grid = np.zeros((c, g, g, g), dtype=np.complex128)
        grid[np.ix_(np.arange(c), pos, pos, pos)] = coil
        z = scipy.fft.fftn(grid, axes=(1, 2, 3), workers=self.workers)
        return z.reshape(c, -1).T

    def interp(self, panel: np.ndarray) -> np.ndarray:
        pr = dense_components(panel.real, self.panel_mode)
        pi = dense_components(panel.imag, self.panel_mode)
        return (self.w @ pr + 1j * (self.w @ pi)).T

    def interp_adjoint(self, samples: np.ndarray) -> np.ndarray:
        panel = np.asarray(samples).T
        pr = dense_components(panel.real, self.panel_mode)
        pi = dense_components(panel.imag, self.panel_mode)
        return (self.wt @ pr + 1j * (self.wt @ pi)).T

    def forward(self, image, smaps) -> np.ndarray:
        return self.interp(self.grid_panel(image, smaps))

    def adjoint_coils(self, samples) -> np.ndarray:
        grid = self.interp_adjoint(samples)
        c, g, pos = grid.shape[0], self.g, self._pos
        vol = scipy.fft.ifftn(grid.reshape(c, g, g, g), axes=(1, 2, 3), workers=self.workers) * float(g ** 3)
        return vol[np.ix_(np.arange(c), pos, pos, pos)] * self.scaling[None]

    def adjoint(self, samples, smaps) -> np.ndarray:
        coil = self.adjoint_coils(samples)
        return np.sum(np.conj(np.asarray(smaps, dtype=np.complex128)) * coil, axis=0)


def cg_sense(forward, adjoint, data, iterations: int, lam: float, operator_scale: float = 1.0):
    """CG on (A^H A + lam) x = A^H y with the operator divided by operator_scale.

    Returns (x, residual history [sqrt(<r,r>)], status dict) with the status
    keys of reference_sparse_solver.py:228-239.
    """
    s = float(operator_scale)
    fwd = (lambda v: forward(v) / s)
    adj = (lambda v: adjoint(v) / s)
    lam_s = lam / (s * s)
    status = {"finite": True, "positive_curvature": True, "completed_iterations": 0,
              "failure": None, "denominators": [], "alphas": []}
    b = adj(np.asarray(data) / s)
    x = np.zeros_like(b)
    if not np.all(np.isfinite(b)):
        status.update(finite=False, failure="nonfinite_rhs")
        return x, [], status
    r = b.copy()
    p = r.copy()
    rs_old = float(np.vdot(r, r).real)
    residuals = [math.sqrt(max(rs_old, 0.0))]
    for iteration in range(iterations):
        ap = adj(fwd(p)) + lam_s * p
        denom = float(np.vdot(p, ap).real)
        status["denominators"].append(denom)
        if not (np.all(np.isfinite(p)) and np.all(np.isfinite(ap)) and math.isfinite(denom)):
            status.update(finite=False, failure=f"nonfinite_iteration_{iteration}")
            break
        if denom <= 0.0:
            status.update(positive_curvature=False, failure=f"nonpositive_curvature_iteration_{iteration}")
            break
        alpha = rs_old / max(denom, 1e-30)
        status["alphas"].append(alpha)
        x = x + alpha * p
        r = r - alpha * ap
        rs_new = float(np.vdot(r, r).real)
        if not (math.isfinite(rs_new) and np.all(np.isfinite(x))):
            status.update(finite=False, failure=f"nonfinite_update_{iteration}")
            break
        residuals.append(math.sqrt(max(rs_new, 0.0)))
        beta = rs_new / max(rs_old, 1e-30)
        p = r + beta * p
        rs_old = rs_new
        status["completed_iterations"] = iteration + 1
    return x, residuals, status


def cg_sense_scheduled(forward, adjoint, ref_forward, ref_adjoint, data, iterations: int, lam: float,
                       scheduled_reference_period: int = 0, explicit_reference_steps=()):
    """CG with scheduled reference steps (reference_sparse_solver.py:200-332, without reliable
    updates): completed iteration s applies the normal operator through ref_forward /
    ref_adjoint when s is a multiple of scheduled_reference_period or listed in
    explicit_reference_steps; the right-hand side comes from ref_adjoint (rhs_adjoint of the
    reference when a reference step is planned).  Returns (x, residual history, status)."""
    steps = frozenset(int(v) for v in explicit_reference_steps)
    status = {"finite": True, "positive_curvature": True, "completed_iterations": 0, "failure": None,
              "scheduled_reference_steps": []}
    b = ref_adjoint(np.asarray(data))
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rs_old = float(np.vdot(r, r).real)
    residuals = [math.sqrt(max(rs_old, 0.0))]
    for iteration in range(iterations):
        done = iteration + 1
        use_ref = done in steps or (scheduled_reference_period > 0 and done % scheduled_reference_period == 0)
        if use_ref:
            ap = ref_adjoint(ref_forward(p)) + lam * p
            status["scheduled_reference_steps"].append(done)
        else:
            ap = adjoint(forward(p)) + lam * p
        denom = float(np.vdot(p, ap).real)
        if not math.isfinite(denom) or denom <= 0.0:
            status.update(positive_curvature=False, failure=f"nonpositive_curvature_iteration_{iteration}")
            break
        alpha = rs_old / max(denom, 1e-30)
        x = x + alpha * p
        r = r - alpha * ap
        rs_new = float(np.vdot(r, r).real)
        residuals.append(math.sqrt(max(rs_new, 0.0)))
        p = r + (rs_new / max(rs_old, 1e-30)) * p
        rs_old = rs_new
        status["completed_iterations"] = done
    return x, residuals, status


def nrmse(candidate, reference) -> float:
    den = max(float(np.linalg.norm(reference)), 1e-30)
    return float(np.linalg.norm(np.asarray(candidate) - np.asarray(reference)) / den)


def magnitude_nrmse(candidate, reference) -> float:
    return nrmse(np.abs(candidate), np.abs(reference))
