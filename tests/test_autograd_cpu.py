"""Hand-written VJPs of the differentiable operators against torch autograd (CPU, FP64).

The operator pieces are a dense FP64 NUDFT matrix here (DenseOps), so the backward
recurrences of trajsparsenufft_b200.autograd are checked exactly (rel <= 1e-9) against
torch.autograd through a plain differentiable implementation of the same steps; the GPU
tests check the same functions on a plan against FP64 finite differences.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from trajsparsenufft_b200 import autograd as tad  # noqa: E402
from trajsparsenufft_b200 import synth  # noqa: E402

N, C = 12, 3


class DenseOps:
    """Coil-wise exact NUDFT as a dense matrix E [M, N*N] (FP64)."""

    def __init__(self, traj, n):
        k = torch.from_numpy(np.asarray(traj, dtype=np.float64))
        idx = torch.arange(n, dtype=torch.float64) - n // 2
        e0 = torch.exp(-2j * np.pi * k[:, 0:1] * idx[None, :])
        e1 = torch.exp(-2j * np.pi * k[:, 1:2] * idx[None, :])
        self.E = (e0[:, :, None] * e1[:, None, :]).reshape(k.shape[0], n * n)
        self.n = n

    def forward_coils(self, ci):
        return ci.reshape(ci.shape[0], -1) @ self.E.T

    def adjoint_coils(self, y):
        return (y @ self.E.conj()).reshape(y.shape[0], self.n, self.n)


def _case(seed=3, density=True):
    g = torch.Generator().manual_seed(seed)
    traj = synth.golden_radial(6, 2 * N)
    ops = DenseOps(traj, N)
    m = traj.shape[0]
    cplx = lambda *s: torch.complex(torch.randn(*s, generator=g, dtype=torch.float64),
                                    torch.randn(*s, generator=g, dtype=torch.float64))
    y = cplx(C, m)
    smaps = cplx(C, N, N) * 0.5
    x0 = cplx(N, N) * 0.1
    xt = cplx(N, N)
    w = torch.rand(m, generator=g, dtype=torch.float64) + 0.5 if density else None
    return ops, y, smaps, x0, xt, w


def _plain_cg(y, smaps, x0, w, ops, lam, iters):
    """The same CG in plain differentiable torch ops."""
    wy = y if w is None else y * w
    G = lambda ci: ops.adjoint_coils(ops.forward_coils(ci) * (1 if w is None else w))
    Mv = lambda v: (smaps.conj() * G(smaps * v)).sum(0) + lam * v
    b = (smaps.conj() * ops.adjoint_coils(wy)).sum(0)
    x = x0
    r = b - Mv(x0)
    p = r
    rho = torch.vdot(r.reshape(-1), r.reshape(-1)).real
    for _ in range(iters):
        q = Mv(p)
        alpha = rho / torch.vdot(p.reshape(-1), q.reshape(-1)).real
        x = x + alpha * p
        r = r - alpha * q
        rho_n = torch.vdot(r.reshape(-1), r.reshape(-1)).real
        p = r + (rho_n / rho) * p
        rho = rho_n
    return x


def _rel(a, b):
    return float((a - b).abs().norm() / max(float(b.abs().norm()), 1e-300))


@pytest.mark.parametrize("checkpoint", [1, 2, 3, 10])
@pytest.mark.parametrize("density", [True, False])
def test_unrolled_cg_vjp_matches_autograd(checkpoint, density):
    ops, y, smaps, x0, xt, w = _case(density=density)
    lam, iters = 0.3, 7
    leaves = [t.clone().requires_grad_(True) for t in (y, smaps, x0)]
    loss = (_plain_cg(*leaves[:3], w, ops, lam, iters) - xt).abs().pow(2).sum()
    ref = torch.autograd.grad(loss, leaves)
    mine_in = [t.clone().requires_grad_(True) for t in (y, smaps, x0)]
    x = tad.cg_sense(mine_in[0], mine_in[1], ops, x0=mine_in[2], density=w, lam=lam, iters=iters,
                     checkpoint=checkpoint)
    loss2 = (x - xt).abs().pow(2).sum()
    got = torch.autograd.grad(loss2, mine_in)
    assert abs(float(loss2.detach()) - float(loss.detach())) <= 1e-10 * float(loss.detach())
    for name, a, b in zip(("y", "smaps", "x0"), got, ref):
        assert _rel(a, b) <= 1e-9, name


def test_zero_initial_image_gradient():
    ops, y, smaps, _, xt, w = _case(seed=5)
    x0 = torch.zeros(N, N, dtype=torch.complex128)
    leaves = [t.clone().requires_grad_(True) for t in (y, smaps, x0)]
    loss = (_plain_cg(*leaves, w, ops, 0.1, 5) - xt).abs().pow(2).sum()
    ref = torch.autograd.grad(loss, leaves)
    mine_in = [t.clone().requires_grad_(True) for t in (y, smaps, x0)]
    loss2 = (tad.cg_sense(mine_in[0], mine_in[1], ops, x0=mine_in[2], density=w, lam=0.1, iters=5) - xt).abs().pow(2).sum()
    got = torch.autograd.grad(loss2, mine_in)
    for name, a, b in zip(("y", "smaps", "x0"), got, ref):
        assert _rel(a, b) <= 1e-9, name


def test_forward_and_adjoint_vjps_match_autograd():
    ops, y, smaps, x0, xt, _ = _case()
    # forward
    xl, sl = x0.clone().requires_grad_(True), smaps.clone().requires_grad_(True)
    yt = torch.complex(torch.randn(y.shape, dtype=torch.float64), torch.randn(y.shape, dtype=torch.float64))
    loss = (ops.forward_coils(sl * xl) - yt).abs().pow(2).sum()
    ref = torch.autograd.grad(loss, (xl, sl))
    xm, sm = x0.clone().requires_grad_(True), smaps.clone().requires_grad_(True)
    got = torch.autograd.grad((tad.nufft_forward(xm, sm, ops) - yt).abs().pow(2).sum(), (xm, sm))
    for a, b in zip(got, ref):
        assert _rel(a, b) <= 1e-10
    # adjoint
    yl, sl = y.clone().requires_grad_(True), smaps.clone().requires_grad_(True)
    loss = ((sl.conj() * ops.adjoint_coils(yl)).sum(0) - xt).abs().pow(2).sum()
    ref = torch.autograd.grad(loss, (yl, sl))
    ym, sm = y.clone().requires_grad_(True), smaps.clone().requires_grad_(True)
    got = torch.autograd.grad((tad.nufft_adjoint(ym, sm, ops) - xt).abs().pow(2).sum(), (ym, sm))
    for a, b in zip(got, ref):
        assert _rel(a, b) <= 1e-10
