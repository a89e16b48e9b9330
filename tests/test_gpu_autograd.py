"""Gradients of the differentiable unrolled CG-SENSE on a GPU plan vs FP64 finite
differences (marked gpu).

loss = |x_10 - x_true|^2 after 10 CG-SENSE iterations from x0 (nonzero).  The gradient with
respect to the k-space data, the coil maps and x0 comes from the hand-written backward
(trajsparsenufft_b200.autograd) on the FP16x2 plan; the reference directional derivatives
are FP64 central finite differences (relative step 1e-6) of the same unrolled CG on the FP64
Kaiser-Bessel oracle operator, over 32 random directions.  Gate: the vector of directional
derivatives agrees within 1e-3 relative.
"""
import numpy as np
import pytest

from gpu_cases import case, measurement
from oracle import operator as oop

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

LAM, ITERS = 1e-4, 10


class _OracleOps:
    def __init__(self, op, n):
        self.op, self.n = op, n

    def forward_coils(self, ci):
        return self.op.forward(np.ones((self.n, self.n)), ci)

    def adjoint_coils(self, y):
        return self.op.adjoint_coils(y)


def _oracle_loss(ops, y, s, x0, xt):
    """The unrolled CG of autograd.UnrolledCgSense in FP64 numpy."""
    G = lambda ci: ops.adjoint_coils(ops.forward_coils(ci))
    Mv = lambda v: (s.conj() * G(s * v)).sum(0) + LAM * v
    b = (s.conj() * ops.adjoint_coils(y)).sum(0)
    x = x0.copy()
    r = b - Mv(x0)
    p = r.copy()
    rho = np.vdot(r, r).real
    for _ in range(ITERS):
        q = Mv(p)
        alpha = rho / np.vdot(p, q).real
        x = x + alpha * p
        r = r - alpha * q
        rho_n = np.vdot(r, r).real
        p = r + (rho_n / rho) * p
        rho = rho_n
    return float(np.sum(np.abs(x - xt) ** 2))


def _fd_check(name, directions):
    """Hand-written gradients of the unrolled CG on the FP16x2 GPU plan against FP64 central
    finite differences of the same unrolled CG on the FP64 KB oracle, along `directions`
    random directions cycling over (y, maps, x0)."""
    from trajsparsenufft_b200 import autograd as tad
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, _ = case(name)
    y = measurement(name).astype(np.complex128)
    rng = np.random.default_rng(17)
    x0 = 0.1 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j)
    ops = tad.PlanOps(plan)
    leaves = [torch.from_numpy(a.astype(np.complex64)).cuda().requires_grad_(True) for a in (y, s, x0)]
    xk = tad.cg_sense(leaves[0], leaves[1], ops, x0=leaves[2], lam=LAM, iters=ITERS, checkpoint=2)
    xt = torch.from_numpy(x).cuda()
    loss = (xk - xt).abs().pow(2).sum()
    loss.backward()
    grads = [t.grad.cpu().numpy().astype(np.complex128) for t in leaves]

    oops = _OracleOps(oop.KbSenseOperator(traj, n, g, j, workers=16), n)
    base = [y, s.astype(np.complex128), x0]
    assert abs(float(loss.detach()) - _oracle_loss(oops, *base, x)) <= 1e-3 * float(loss.detach())
    got, want = [], []
    for k in range(directions):
        v = k % 3
        d = rng.standard_normal(base[v].shape) + 1j * rng.standard_normal(base[v].shape)
        eps = 1e-6 * np.linalg.norm(base[v]) / np.linalg.norm(d)
        plus = [a.copy() for a in base]
        minus = [a.copy() for a in base]
        plus[v] = plus[v] + eps * d
        minus[v] = minus[v] - eps * d
        fd = (_oracle_loss(oops, *plus, x) - _oracle_loss(oops, *minus, x)) / (2 * eps)
        got.append(float(np.vdot(grads[v], d).real))
        want.append(fd)
    got, want = np.array(got), np.array(want)
    assert np.linalg.norm(got - want) <= 1e-3 * np.linalg.norm(want)
    for v in range(3):  # each input's directional derivatives on their own
        sel = np.arange(v, directions, 3)
        assert np.linalg.norm(got[sel] - want[sel]) <= 1e-3 * np.linalg.norm(want[sel]), v


def test_unrolled_cg_gradients_match_fp64_finite_differences():
    """64^2 image, 4 coils: 32 directions."""
    _fd_check("small", 32)


def test_unrolled_cg_gradients_match_fp64_finite_differences_grad4_shape():
    """One case of the differentiable configuration (256^2 image, 512^2 grid, 8 coils,
    golden-angle radial 128 x 512, 10 iterations, checkpoint every 2): 9 directions, three per
    input, since every FP64 oracle evaluation is a full 10-iteration CG at this size."""
    _fd_check("grad4", 9)


def test_differentiable_forward_matches_graph_solver():
    """From x0 = 0 the differentiable solve reproduces tsn_cg_sense (same FP16x2 operator)."""
    from trajsparsenufft_b200 import autograd as tad
    from trajsparsenufft_b200.operator import Plan
    from gpu_cases import torch_inputs
    traj, x, s, n, g, c, j, _ = case("cfg0")
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j)
    _, st, yt = torch_inputs("cfg0")
    x_graph, _, _ = plan.cg_sense(yt, st, lam=LAM, iters=ITERS)
    with torch.no_grad():
        x_diff = tad.cg_sense(yt, st, tad.PlanOps(plan), lam=LAM, iters=ITERS)
    rel = float((x_diff - x_graph).abs().norm() / x_graph.abs().norm())
    assert rel <= 1e-4


def test_graph_captured_gradient_step_matches_eager():
    """The whole differentiable step (forward solve, loss, backward) captured as one CUDA graph
    gives the eager step's gradients; replays with new inputs in the static tensors follow them."""
    from trajsparsenufft_b200 import autograd as tad
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, _ = case("small")
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j)
    ops = tad.PlanOps(plan)
    y0 = torch.from_numpy(measurement("small")).cuda()
    s0 = torch.from_numpy(s).cuda()
    xt = torch.from_numpy(x).cuda()

    def eager(y, smaps):
        yl = y.detach().clone().requires_grad_(True)
        sl = smaps.detach().clone().requires_grad_(True)
        x0 = torch.zeros((n, n), dtype=torch.complex64, device="cuda", requires_grad=True)
        loss = (tad.cg_sense(yl, sl, ops, x0=x0, lam=LAM, iters=ITERS, checkpoint=2) - xt).abs().pow(2).sum()
        loss.backward()
        return loss.detach(), [yl.grad, sl.grad, x0.grad]

    y_st, s_st = y0.clone(), s0.clone()
    leaves = [y_st.detach().requires_grad_(True), s_st.detach().requires_grad_(True),
              torch.zeros((n, n), dtype=torch.complex64, device="cuda", requires_grad=True)]

    def body():
        yl, sl, x0 = leaves
        loss = (tad.cg_sense(yl, sl, ops, x0=x0, x0_zero=True, lam=LAM, iters=ITERS, checkpoint=2)
                - xt).abs().pow(2).sum()
        loss.backward()
        return loss

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(2):
            for leaf in leaves:
                leaf.grad = None
            body()
    torch.cuda.current_stream().wait_stream(side)
    for leaf in leaves:
        leaf.grad = None
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, capture_error_mode="relaxed"):
        loss_g = body()
    for scale in (1.0, 0.5):
        y_st.copy_(y0 * scale)
        graph.replay()
        loss_e, grads_e = eager(y0 * scale, s0)
        torch.cuda.synchronize()
        assert torch.allclose(loss_g, loss_e, rtol=1e-6, atol=0)
        for leaf, ge in zip(leaves, grads_e):
            rel = float(torch.linalg.vector_norm(leaf.grad - ge) / torch.linalg.vector_norm(ge))
            assert rel <= 1e-6, rel


def test_normal_operator_and_fp64_dots_in_cuda():
    """tsn_normal (q = sum_c conj(S_c) F^H W F(S_c p) + lam p with its coil images and FP64
    Re <p, q>) and tsn_rdot, which the differentiable CG uses on a GPU plan, against the same
    operator composed from tsn_forward / tsn_adjoint on coil images with torch (the generic
    path of autograd._Sense) and against the FP16x2 oracle emulation.  Gates: q and the coil
    images within 2e-5 rel of both (FP16x2 rounding; the fused path scales its panel by |p|
    instead of |S p|); the FP64 inner products within 1e-12 rel of numpy's over the same
    FP32 vectors; a lazily conjugated view is refused."""
    from trajsparsenufft_b200 import synth
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, readout = case("grad4")
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j)
    w = synth.ramp_density(traj, readout).astype(np.float32)
    rng = np.random.default_rng(9)
    p = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    pt, st, wt = torch.from_numpy(p).cuda(), torch.from_numpy(s).cuda(), torch.from_numpy(w).cuda()
    for _ in range(2):  # repeated calls on one plan: the workspaces carry nothing over
        q, t, pq = plan.normal(pt, st, density=wt, lam=LAM, coils=True, pq=True)
        torch.cuda.synchronize()
    t_ref = plan.adjoint(plan.forward((st * pt).contiguous()) * wt)
    q_ref = (st.conj() * t_ref).sum(0) + LAM * pt
    qn, tn = q.cpu().numpy(), t.cpu().numpy()
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    assert rel(qn, q_ref.cpu().numpy()) <= 2e-5
    assert rel(tn, t_ref.cpu().numpy()) <= 2e-5
    emu = oop.KbSenseOperator(traj, n, g, j, matrix_mode="fp16", panel_mode="split2", workers=8)
    q_emu = emu.adjoint(emu.forward(p.astype(np.complex128), s) * w, s) + LAM * p
    assert rel(qn, q_emu) <= 2e-5
    want = float(np.sum(p.real.astype(np.float64) * qn.real + p.imag.astype(np.float64) * qn.imag))
    assert abs(float(pq.cpu()) - want) <= 1e-12 * abs(want)
    q2, _, _ = plan.normal(pt, st, density=wt, lam=LAM)
    np.testing.assert_array_equal(q2.cpu().numpy(), qn)  # without the extra outputs: the same q
    d = plan.rdot(pt, q)
    assert abs(float(d.cpu()) - want) <= 1e-12 * abs(want)
    with pytest.raises(ValueError):
        plan.rdot(pt.conj(), q)


class _ComposedOps:
    """PlanOps without its fused pieces: autograd._Sense then composes the SENSE algebra, the
    inner products and the reverse CG recurrences from the coil operators with torch."""

    def __init__(self, plan):
        self.plan = plan

    def forward_coils(self, ci):
        return self.plan.forward(ci.contiguous())

    def adjoint_coils(self, y):
        return self.plan.adjoint(y.contiguous())


def test_fused_backward_matches_composed_backward():
    """The gradients through the plan's kernels (tsn_normal, tsn_rdot, tsn_cg_adjoint_step /
    _finish) against the same unrolled CG composed with torch from the coil operators, at the
    grad4 shape with density weights and a nonzero x0. Gate: 1e-3 relative per input (the two
    paths round the FP16x2 panels differently and the 10-iteration CG amplifies it; the FD
    checks hold both to the FP64 truth at the same 1e-3)."""
    from trajsparsenufft_b200 import autograd as tad
    from trajsparsenufft_b200 import synth
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, readout = case("grad4")
    y = measurement("grad4")
    w = torch.from_numpy(synth.ramp_density(traj, readout).astype(np.float32)).cuda()
    rng = np.random.default_rng(23)
    x0 = (0.1 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))).astype(np.complex64)
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j)
    xt = torch.from_numpy(x).cuda()
    grads = []
    for ops in (tad.PlanOps(plan), _ComposedOps(plan)):
        leaves = [torch.from_numpy(a.astype(np.complex64)).cuda().requires_grad_(True) for a in (y, s, x0)]
        xk = tad.cg_sense(leaves[0], leaves[1], ops, x0=leaves[2], density=w, lam=LAM, iters=ITERS, checkpoint=2)
        (xk - xt).abs().pow(2).sum().backward()
        grads.append([t.grad.cpu().numpy() for t in leaves])
    for a, b in zip(*grads):
        assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b)
