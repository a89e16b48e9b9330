"""Differentiable NUFFT forward / adjoint and unrolled CG-SENSE (torch.autograd.Function).

The operator pieces come from a `CoilOps` object: the coil-wise NUFFT F (coil images
[C][N][N] -> samples [C][M]) and its adjoint F^H, both linear.  `PlanOps` serves them from a
GPU plan (tsn_forward / tsn_adjoint with smaps = NULL); any object with the same two methods
works (the CPU tests use a dense FP64 matrix).  With S the coil maps, W the density weights
and G = F^H W F coil by coil:

    A x      = F(S x)                       forward
    A^H y    = sum_c conj(S_c) F^H(y_c)     adjoint
    M p      = sum_c conj(S_c) G(S_c p) + lam p

Gradients follow PyTorch's complex convention (dL = Re<grad, dz>).  For w = S u (linear in
S) the map gradient is grad_w conj(u); for w = conj(S) u it is conj(grad_w) u.

The unrolled solve is the reference's CG (launch_cg, nufft_fp16x2_cg_bench.cu:241-268;
reference_sparse_solver.py cg_sense) from an initial image x0:
    r0 = A^H W y - M x0,  p0 = r0,  rho_k = |r_k|^2
    q = M p, alpha = rho / Re<p, q>, x += alpha p, r -= alpha q, beta = rho'/rho, p = r + beta p.
Backward runs the adjoint recurrences of these steps in reverse, restarting each segment from
a checkpoint (x, r, p, rho) stored every `checkpoint` iterations, and returns gradients for
the k-space data y, the coil maps and x0.  A checkpoint also keeps q = M p of its own step
(and the coil images G(S p) when the maps need gradients), which the forward computed anyway,
so a segment recomputes `checkpoint - 1` forward steps.  Each reverse step applies G once per
coil for the adjoint of q = M p, which also yields the coil-map term.
"""

from __future__ import annotations

import torch


class PlanOps:
    """Coil-wise NUFFT pieces from a GPU plan (FP16x2 sparse interpolation, FP32 FFTs)."""

    def __init__(self, plan):
        self.plan = plan

    def forward_coils(self, coil_images: torch.Tensor) -> torch.Tensor:
        return self.plan.forward(coil_images.contiguous())

    def adjoint_coils(self, y: torch.Tensor) -> torch.Tensor:
        return self.plan.adjoint(y.contiguous())

    def normal(self, p, smaps, density, lam, coils=False, pq=False, p_parts=None):
        """(sum_c conj(S_c) G(S_c p) + lam p, the coil images G(S_c p) or None, Re <p, q> or
        None) in the plan's kernels (tsn_normal): SENSE expansion, weighting, combine and the
        FP64 inner product fused into the NUFFT stages. p_parts: FP64 partials of |p|^2 from
        the CG step that made p."""
        return self.plan.normal(p.contiguous(), smaps.contiguous(), density=density, lam=lam, coils=coils, pq=pq,
                                p_norm_parts=p_parts)

    def rdot(self, a, b):
        """Re <a, b> in FP64, fixed order (tsn_rdot), as a 0-d device tensor."""
        return self.plan.rdot(a.contiguous(), b.contiguous())

    def forward_maps(self, x, smaps):
        """F(S_c x) with the SENSE expansion inside the row transforms (tsn_forward)."""
        return self.plan.forward(x.contiguous(), smaps.contiguous())

    def step(self, rho, gamma, x, p, r, q):
        """One CG step in the plan's kernels: (x' or None, r', p', rho', |p'|^2 partials)."""
        return self.plan.cg_step(rho, gamma, None if x is None else x.contiguous(), p.contiguous(), r.contiguous(),
                                 q.contiguous(), norm_parts=True)

    def adjoint_step(self, rho, rho_n, gamma, rhob, rb, pb, p, q, r_n, xb):
        """Reverse-mode CG step in the plan's kernels (rb, pb in place): (qb, rhob of the step,
        |qb|^2 partials)."""
        return self.plan.cg_adjoint_step(rho, rho_n, gamma, rhob, rb, pb, p, q, r_n, xb, norm_parts=True)

    def adjoint_finish(self, pb, mqb, qb=None, t=None, tb=None, p=None, sb=None):
        """pb += M qb and the coil-map cotangent update, in place."""
        self.plan.cg_adjoint_finish(pb, mqb, qb, t, tb, p, sb)


def _rdot(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """Re <a, b> = sum(a.re b.re + a.im b.im), accumulated in FP64 (a 0-d tensor), like the graph
    solver's CG inner products (a complex64 vdot would accumulate in FP32)."""
    ar = torch.view_as_real(a.reshape(-1)).reshape(-1).to(torch.float64)
    br = torch.view_as_real(b.reshape(-1)).reshape(-1).to(torch.float64)
    return torch.dot(ar, br)


class _Sense:
    """SENSE algebra over a CoilOps object (no autograd inside).  When the ops object has
    `normal` and `rdot` (PlanOps), M p, its coil images and the FP64 inner products run in the
    plan's CUDA kernels; otherwise they are composed here from forward_coils / adjoint_coils."""

    def __init__(self, ops, smaps, density, lam):
        self.ops, self.s, self.w, self.lam = ops, smaps, density, lam
        self.fused = all(hasattr(ops, k) for k in ("normal", "rdot", "forward_maps", "step", "adjoint_step",
                                                   "adjoint_finish"))

    def weigh(self, y):
        return y if self.w is None else y * self.w

    def G(self, coils):
        return self.ops.adjoint_coils(self.weigh(self.ops.forward_coils(coils)))

    def combine(self, coils):
        return (self.s.conj() * coils).sum(0)

    def dot(self, a, b):
        return self.ops.rdot(a, b) if self.fused else _rdot(a, b)

    def A(self, x):
        """F(S x), the coil k-space of image x."""
        return self.ops.forward_maps(x, self.s) if self.fused else self.ops.forward_coils(self.s * x)

    # `parts` below: FP64 partial sums of |p|^2 that the fused CG steps hand to the next
    # normal-operator application (its panel scale); None computes them there.
    def M(self, p, parts=None):
        if self.fused:
            return self.ops.normal(p, self.s, self.w, self.lam, p_parts=parts)[0]
        return self.combine(self.G(self.s * p)) + self.lam * p

    def M_dot(self, p, parts=None):
        """(M p, Re <p, M p>)."""
        if self.fused:
            q, _, pq = self.ops.normal(p, self.s, self.w, self.lam, pq=True, p_parts=parts)
            return q, pq
        q = self.M(p)
        return q, _rdot(p, q)

    def M_coils_dot(self, p, parts=None):
        """(M p, the coil images G(S p), Re <p, M p>)."""
        if self.fused:
            return self.ops.normal(p, self.s, self.w, self.lam, coils=True, pq=True, p_parts=parts)
        q, t = self.M_coils(p)
        return q, t, _rdot(p, q)

    def step(self, rho, gamma, x, p, r, q):
        """CG step: (x + alpha p or None, r' = r - alpha q, p' = r' + (rho'/rho) p, rho' = |r'|^2,
        the |p'|^2 partials or None) with alpha = rho / gamma."""
        if self.fused:
            return self.ops.step(rho, gamma, x, p, r, q)
        alpha = rho / gamma
        x_n = None if x is None else x + alpha * p
        r_n = r - alpha * q
        rho_n = _rdot(r_n, r_n)
        return x_n, r_n, r_n + (rho_n / rho) * p, rho_n, None

    def M_coils(self, p, parts=None):
        """(M p, the coil images G(S p)) — the second feeds the coil-map gradient."""
        if self.fused:
            q, t, _ = self.ops.normal(p, self.s, self.w, self.lam, coils=True, p_parts=parts)
            return q, t
        t = self.G(self.s * p)
        return self.combine(t) + self.lam * p, t


class NufftForward(torch.autograd.Function):
    """y = A x = F(S x)."""

    @staticmethod
    def forward(ctx, x, smaps, ops):
        ctx.save_for_backward(x, smaps)
        ctx.ops = ops
        return ops.forward_coils(smaps * x)

    @staticmethod
    def backward(ctx, gy):
        x, smaps = ctx.saved_tensors
        u = ctx.ops.adjoint_coils(gy)
        gx = (smaps.conj() * u).sum(0) if ctx.needs_input_grad[0] else None
        gs = u * x.conj() if ctx.needs_input_grad[1] else None
        return gx, gs, None


class NufftAdjoint(torch.autograd.Function):
    """x = A^H y = sum_c conj(S_c) F^H(y_c)."""

    @staticmethod
    def forward(ctx, y, smaps, ops):
        u = ops.adjoint_coils(y)
        ctx.save_for_backward(smaps, u)
        ctx.ops = ops
        return (smaps.conj() * u).sum(0)

    @staticmethod
    def backward(ctx, gx):
        smaps, u = ctx.saved_tensors
        gy = ctx.ops.forward_coils(smaps * gx) if ctx.needs_input_grad[0] else None
        gs = gx.conj() * u if ctx.needs_input_grad[1] else None
        return gy, gs, None


def nufft_forward(x, smaps, ops):
    return NufftForward.apply(x, smaps, ops)


def nufft_adjoint(y, smaps, ops):
    return NufftAdjoint.apply(y, smaps, ops)


class UnrolledCgSense(torch.autograd.Function):
    """x_K of `iters` CG-SENSE iterations from x0; differentiable in y, smaps and x0."""

    @staticmethod
    def forward(ctx, y, smaps, x0, density, ops, lam, iters, checkpoint, x0_zero):
        S = _Sense(ops, smaps, density, lam)
        u = ops.adjoint_coils(S.weigh(y))          # F^H W y, coil images
        b = S.combine(u)
        if x0_zero is None:                        # decided from the values (a host sync)
            x0_zero = not bool(x0.abs().amax() > 0)
        x = x0.clone()
        r = b.clone() if x0_zero else b - S.M(x0)
        p = r.clone()
        rho = S.dot(r, r)
        cps = [(x, r, p, rho)]
        need_s = ctx.needs_input_grad[1]
        firsts = []   # q = M p (and the coil images G(S p) when maps need gradients) of each
        parts = None
        for k in range(iters):   # checkpointed step: the backward reuses them instead of recomputing
            if k % checkpoint == 0 and need_s:
                q, t, gamma = S.M_coils_dot(p, parts)
                firsts.append((q, t))
            else:
                q, gamma = S.M_dot(p, parts)
                if k % checkpoint == 0:
                    firsts.append((q,))
            x, r, p, rho, parts = S.step(rho, gamma, x, p, r, q)
            if (k + 1) % checkpoint == 0 and k + 1 < iters:
                cps.append((x, r, p, rho))
        ctx.ops, ctx.lam, ctx.iters, ctx.checkpoint, ctx.x0_zero = ops, lam, iters, checkpoint, x0_zero
        ctx.has_density = density is not None
        ctx.first_width = 2 if need_s else 1
        flat = [v for cp in cps for v in cp] + [v for f in firsts for v in f]
        ctx.save_for_backward(smaps, x0, u, *(() if density is None else (density,)), *flat)
        return x

    @staticmethod
    def backward(ctx, gx):
        saved = ctx.saved_tensors
        smaps, x0, u = saved[0], saved[1], saved[2]
        density = saved[3] if ctx.has_density else None
        flat = saved[4 if ctx.has_density else 3:]
        n_seg = (ctx.iters + ctx.checkpoint - 1) // ctx.checkpoint   # segments (firsts)
        n_cp = max(1, n_seg)                                          # checkpoints incl. the start
        cps = [tuple(flat[i:i + 4]) for i in range(0, 4 * n_cp, 4)]
        fw = ctx.first_width
        firsts = [tuple(flat[4 * n_cp + i:4 * n_cp + i + fw]) for i in range(0, fw * n_seg, fw)]
        S = _Sense(ctx.ops, smaps, density, ctx.lam)
        need_y, need_s, need_x0 = ctx.needs_input_grad[0], ctx.needs_input_grad[1], ctx.needs_input_grad[2]
        c, iters = ctx.checkpoint, ctx.iters
        xb = gx.contiguous()
        rb = torch.zeros_like(xb)
        pb = torch.zeros_like(xb)
        rhob = torch.zeros((), dtype=torch.float64, device=gx.device)
        sb = torch.zeros_like(smaps) if need_s else None
        for seg in reversed(range(len(cps))):
            k0, k1 = seg * c, min(seg * c + c, iters)
            _, r, p, rho = cps[seg]
            steps = []
            parts = None
            for k in range(k0, k1):  # recompute this segment's forward states
                if k == k0:          # kept by the forward with the checkpoint
                    q, t = firsts[seg][0], (firsts[seg][1] if need_s else None)
                elif need_s:
                    q, t = S.M_coils(p, parts)
                else:
                    q, t = S.M(p, parts), None
                gamma = S.dot(p, q)
                _, r_n, p_n, rho_n, parts = S.step(rho, gamma, None, p, r, q)
                ab = (None, None) if S.fused else (rho / gamma, rho_n / rho)  # alpha, beta: composed path
                steps.append((p, q, t, r_n, rho, rho_n, gamma, *ab))
                p = p_n
                r, rho = r_n, rho_n
            for p, q, t, r_n, rho, rho_n, gamma, alpha, beta in reversed(steps):
                if S.fused:  # the same recurrences in the plan's kernels (rb, pb, sb in place)
                    qb, rhob, qparts = ctx.ops.adjoint_step(rho, rho_n, gamma, rhob, rb, pb, p, q, r_n, xb)
                    if need_s:
                        mqb, tb = S.M_coils(qb, qparts)
                        ctx.ops.adjoint_finish(pb, mqb, qb, t, tb, p, sb)
                    else:
                        ctx.ops.adjoint_finish(pb, S.M(qb, qparts))
                    continue
                rb = rb + pb                                   # p' = r' + beta p
                betab = S.dot(pb, p)
                pbk = beta * pb
                rhob_n = rhob + betab / rho                    # beta = rho' / rho
                rhobk = -betab * rho_n / (rho * rho)
                rb = rb + (2.0 * rhob_n) * r_n                 # rho' = |r'|^2
                qb = -alpha * rb                               # r' = r - alpha q
                alphab = -S.dot(rb, q)
                pbk = pbk + alpha * xb                         # x' = x + alpha p
                alphab = alphab + S.dot(xb, p)
                rhobk = rhobk + alphab / gamma                 # alpha = rho / gamma
                gammab = -alphab * rho / (gamma * gamma)
                pbk = pbk + gammab * q                         # gamma = Re <p, q>
                qb = qb + gammab * p
                if need_s:                                     # q = M p (M Hermitian)
                    mqb, tb = S.M_coils(qb)
                    sb = sb + qb.conj() * t + tb * p.conj()
                else:
                    mqb = S.M(qb)
                pb = pbk + mqb
                rhob = rhobk
        # p0 = r0, rho0 = |r0|^2, r0 = b - M x0
        r0 = cps[0][1]
        rb = rb + pb + (2.0 * rhob) * r0
        gy = gs = gx0 = None
        if need_x0:
            gx0 = xb - S.M(rb)                                # x0 directly and through r0 = b - M x0
        if need_s:
            if not ctx.x0_zero:                               # the - M x0 term, cotangent -rb
                v = -rb
                sb = sb + v.conj() * S.G(smaps * x0) + S.G(smaps * v) * x0.conj()
            sb = sb + rb.conj() * u                           # b = sum conj(S) F^H W y
            gs = sb
        if need_y:
            gy = S.weigh(S.A(rb))
        return gy, gs, gx0, None, None, None, None, None, None


def cg_sense(y, smaps, ops, *, x0=None, density=None, lam=1e-4, iters=10, checkpoint=2, x0_zero=None):
    """Differentiable unrolled CG-SENSE: x after `iters` iterations of (A^H W A + lam) x = A^H W y
    from x0 (zero by default), with CG states checkpointed every `checkpoint` iterations.

    x0_zero states whether x0 is all zeros (which saves one operator application); None
    decides it from x0's values, a device-to-host read that a CUDA-graph capture of the step
    cannot contain, so graph-captured steps pass it explicitly."""
    if x0 is None:
        x0 = torch.zeros(smaps.shape[1:], dtype=smaps.dtype, device=smaps.device)
        x0_zero = True
    if checkpoint < 1:
        raise ValueError("checkpoint interval must be >= 1")
    return UnrolledCgSense.apply(y, smaps, x0, density, ops, float(lam), int(iters), int(checkpoint),
                                 None if x0_zero is None else bool(x0_zero))
