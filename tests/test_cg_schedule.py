"""The device CG's scalar schedule, restated on the host, against the oracle's CG.

The GPU solve finishes iteration k-1's update inside iteration k's forward rows: the inverse
rows write per-line FP64 partials of <p, Ap>, Re <r, Ap>, <Ap, Ap> and <r, r>, and the next
forward rows take rho = <r, r> (direct, like the reference's rs_old), alpha = rho / <p, Ap>
and rho' = rho - 2 alpha Re <r, Ap> + alpha^2 <Ap, Ap> before x += alpha p, r -= alpha Ap,
p = r + beta p. Only the last iteration (and one before a reliable residual) computes rho'
directly from the updated r. This restatement keeps the device's precisions (FP32 vectors,
FP64 per-line partials summed in order) and must track the oracle's CG
(oracle/operator.py:cg_sense, reference_sparse_solver.py:297-323) on a small system.
"""
import numpy as np

from oracle import operator as oop


def _line_dots(a, b, n):
    """FP64 per-line partials of Re <a, b> over lines of n values, summed in line order."""
    prod = (a.real.astype(np.float64) * b.real + a.imag.astype(np.float64) * b.imag).reshape(-1, n)
    return float(np.sum(prod.sum(axis=1)))


def _fused_cg(normal, b, iters, n):
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rho = _line_dots(r, r, n)
    hist = [rho]
    expansion_vs_direct = []
    for k in range(iters):
        ap = normal(p).astype(np.complex64)
        pap = _line_dots(p, ap, n)
        if k > 0:  # the forward rows of iteration k+1 read <r, r> of the stored r directly
            rho = _line_dots(r, r, n)
            hist[k] = rho
        alpha = rho / pap if pap > 0 else 0.0
        af = np.float32(alpha)
        if k + 1 < iters:  # finished by the next forward rows
            rap, apap = _line_dots(r, ap, n), _line_dots(ap, ap, n)
            rho_new = max(rho - 2.0 * alpha * rap + alpha * alpha * apap, 0.0)
            x = (x + af * p).astype(np.complex64)
            r = (r - af * ap).astype(np.complex64)
            expansion_vs_direct.append(abs(rho_new - _line_dots(r, r, n)) / _line_dots(r, r, n))
            beta = np.float32(rho_new / max(rho, 1e-30))
            p = (r + beta * p).astype(np.complex64)
        else:  # cg_update: direct residual norm
            x = (x + af * p).astype(np.complex64)
            r = (r - af * ap).astype(np.complex64)
            rho_new = _line_dots(r, r, n)
        hist.append(rho_new)
        rho = rho_new
    return x, hist, expansion_vs_direct


def test_fused_update_tracks_the_oracle_cg():
    rng = np.random.default_rng(20260823)
    n, m, lam = 16, 600, 1e-2
    a = (rng.standard_normal((m, n * n)) + 1j * rng.standard_normal((m, n * n))) / np.sqrt(m)
    y = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    normal = (lambda v: a.conj().T @ (a @ v) + lam * v)
    b = (a.conj().T @ y).astype(np.complex64)
    iters = 10
    x_ref, res_ref, status = oop.cg_sense(lambda v: a @ v, lambda v: a.conj().T @ v, y, iters, lam)
    assert status["completed_iterations"] == iters
    x, hist, _ = _fused_cg(normal, b, iters, n)
    # residual history: the expansion form agrees with the direct one to FP32 vector rounding
    np.testing.assert_allclose(np.sqrt(hist), res_ref, rtol=2e-4)
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < 1e-4
    assert hist[-1] < 1e-2 * hist[0]


def test_expanded_rho_does_not_drift_on_long_solves():
    """Over 60 iterations the residual falls by many orders of magnitude; because every
    expansion restarts from the direct <r, r> of the stored FP32 residual, the expanded rho'
    stays within FP32 rounding of |r'|^2 of the stored vector (it would drift if the
    expansion were carried from one iteration to the next)."""
    rng = np.random.default_rng(7)
    n, m, lam = 12, 400, 5e-2
    a = (rng.standard_normal((m, n * n)) + 1j * rng.standard_normal((m, n * n))) / np.sqrt(m)
    y = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    normal = (lambda v: a.conj().T @ (a @ v) + lam * v)
    b = (a.conj().T @ y).astype(np.complex64)
    x, hist, rel = _fused_cg(normal, b, 60, n)
    assert hist[-1] < 1e-8 * hist[0]
    assert max(rel) < 1e-3


def test_scheduled_reference_steps_oracle():
    """oracle cg_sense_scheduled (reference_sparse_solver.py:249-260): completed iterations that
    are multiples of the period or listed explicitly take the reference operator; with the same
    operator on both sides it is the plain CG, and with every step on the reference operator it
    is the plain CG of that operator (its right-hand side included)."""
    rng = np.random.default_rng(3)
    n = 24
    a = rng.standard_normal((40, n)) + 1j * rng.standard_normal((40, n))
    a_low = (a + 1e-3 * rng.standard_normal(a.shape)).astype(np.complex128)
    data = rng.standard_normal(40) + 1j * rng.standard_normal(40)
    fwd, adj = (lambda v: a_low @ v), (lambda v: a_low.conj().T @ v)
    rfwd, radj = (lambda v: a @ v), (lambda v: a.conj().T @ v)
    x0, h0, s0 = oop.cg_sense(fwd, adj, data, 8, 1e-3)
    x1, h1, s1 = oop.cg_sense_scheduled(fwd, adj, fwd, adj, data, 8, 1e-3, scheduled_reference_period=2)
    np.testing.assert_allclose(x1, x0, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(h1, h0, rtol=1e-12)
    assert s1["scheduled_reference_steps"] == [2, 4, 6, 8]
    xr, hr, _ = oop.cg_sense(rfwd, radj, data, 8, 1e-3)
    x2, h2, _ = oop.cg_sense_scheduled(fwd, adj, rfwd, radj, data, 8, 1e-3, scheduled_reference_period=1)
    np.testing.assert_allclose(x2, xr, rtol=1e-12, atol=1e-12)
    _, _, s3 = oop.cg_sense_scheduled(fwd, adj, rfwd, radj, data, 8, 1e-3, scheduled_reference_period=3,
                                      explicit_reference_steps=(5, 7))
    assert s3["scheduled_reference_steps"] == [3, 5, 6, 7]
