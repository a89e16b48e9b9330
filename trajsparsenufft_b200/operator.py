"""Plans and operators: the Python face of the C ABI.

``Plan`` mirrors what the reference CG binary assembles from its argv
(nufft_fp16x2_cg_bench.cu:279-297: four pack directories, a runtime directory,
the operator scale, the iteration count) plus the forward / adjoint operator
pair of nufft_integrated_bench.cu:604-674.  Device memory and streams come from
torch (plumbing only); every operator runs in the CUDA library, there is no
CPU or torch fallback.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import CgStatus, PlanDesc, PlanInfo, check, lib, ptr


def _torch():
    import torch
    return torch


def _stream_handle(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dev_ptr(t, dtype, shape, name):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if t.is_complex() and t.is_conj():
        raise ValueError(f"{name} is a lazily conjugated view: pass {name}.resolve_conj()")
    return C.c_void_p(t.data_ptr())


INTERP = {"auto": 0, "mma_sp": 1, "tcgen05": 2}


def plan_desc(im_size=256, grid_size=512, coils=8, width=6, planner="optimized", policy="morton",
              seed=20260823, threads=0, reference_layout=False, device=None, dims=2, interp="auto") -> PlanDesc:
    d = PlanDesc()
    check(lib().tsn_plan_desc_default(C.byref(d)))
    d.interp = INTERP[interp]
    d.im_size, d.grid_size, d.coils, d.kernel_width = im_size, grid_size, coils, width
    d.dims = int(dims)
    d.planner, d.policy, d.seed, d.threads = _lib.PLANNER[planner], _lib.POLICY[policy], seed, threads
    d.flags = _lib.FLAG_REFERENCE_LAYOUT if reference_layout else 0
    if device is None:
        try:
            torch = _torch()
            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        except Exception:
            device = 0
    d.device = int(device)
    return d


class Plan:
    """Device-resident forward/adjoint packs of one trajectory plus solver workspaces."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        info = PlanInfo()
        check(lib().tsn_plan_get_info(self._h, C.byref(info)))
        self.samples = info.samples
        self.im_size = info.im_size
        self.grid_size = info.grid_size
        self.coils = info.coils
        self.width = info.kernel_width
        self.components = info.components
        self.dims = info.dims if info.dims in (2, 3) else 2
        self.info = {
            "samples": info.samples, "im_size": info.im_size, "grid_size": info.grid_size, "coils": info.coils,
            "kernel_width": info.kernel_width, "components": info.components,
            "groups": list(info.groups), "tiles": list(info.tiles), "active_rows": list(info.active_rows),
            "nnz": list(info.nnz), "pack_bytes": list(info.pack_bytes), "workspace_bytes": info.workspace_bytes,
            "plan_seconds": info.plan_seconds, "interp": info.interp, "dims": self.dims,
        }
        self.interp = {v: k for k, v in INTERP.items()}.get(info.interp, str(info.interp))

    def device_error(self) -> int:
        """Nonzero once a tensor-core interpolation launch of this plan gave up a bounded wait
        (read at call time: synchronize the plan's streams first)."""
        info = PlanInfo()
        check(lib().tsn_plan_get_info(self._h, C.byref(info)))
        return int(info.device_error)

    # ---- construction ------------------------------------------------------------------
    @classmethod
    def from_trajectory(cls, trajectory, *, im_size=256, grid_size=512, coils=8, width=6, planner="optimized",
                        policy="morton", seed=20260823, threads=0, reference_layout=False, device=None,
                        interp="auto", reference_steps=False) -> "Plan":
        """Pack a trajectory once (C++ planner) and upload both views.  interp chooses the sparse
        interpolation kernel: "mma_sp" (warp mma.sp per 16-row tile), "tcgen05" (tcgen05.mma.sp
        with stacked tiles; real-coefficient pack with 8 coils) or "auto".  reference_steps
        keeps an FP32-class copy of the operator (coefficients as FP16 high + FP16 residual) for
        the CG's scheduled reference steps (TSN_FLAG_REFERENCE_STEPS)."""
        traj = np.asarray(trajectory, dtype=np.float32)
        dims = 3 if traj.ndim == 2 and traj.shape[1] == 3 else 2
        t = np.ascontiguousarray(traj.reshape(-1, dims))
        d = plan_desc(im_size, grid_size, coils, width, planner, policy, seed, threads, reference_layout, device, dims,
                      interp)
        if reference_steps:
            d.flags |= _lib.FLAG_REFERENCE_STEPS
        h = C.c_void_p()
        check(lib().tsn_plan_create_from_trajectory(ptr(t, C.c_float), t.shape[0], C.byref(d), C.byref(h)))
        return cls(h)

    @classmethod
    def from_pack(cls, fwd_real, fwd_imag, adj_real, adj_imag, *, im_size=256, grid_size=512, coils=8, width=6,
                  scaling=None, device=None) -> "Plan":
        """Load reference-format pack directories (load_direction x 2)."""
        enc = (lambda p: None if p is None else str(Path(p)).encode())
        sc = None if scaling is None else np.ascontiguousarray(np.asarray(scaling, dtype=np.float32))
        if sc is not None and sc.shape != (im_size, im_size):
            raise ValueError("scaling must be [im_size, im_size]")
        d = plan_desc(im_size, grid_size, coils, width, device=device)
        h = C.c_void_p()
        check(lib().tsn_plan_create_from_pack(enc(fwd_real), enc(fwd_imag), enc(adj_real), enc(adj_imag),
                                              ptr(sc, C.c_float), C.byref(d), C.byref(h)))
        return cls(h)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().tsn_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- operators ------------------------------------------------------------------------
    @property
    def image_shape(self) -> tuple:
        """[N, N] for image plans, [N, N, N] for volume plans."""
        return (self.im_size,) * self.dims

    @property
    def maps_shape(self) -> tuple:
        return (self.coils,) + self.image_shape

    @property
    def grid_cells(self) -> int:
        return self.grid_size ** self.dims

    def _image_shape(self, smaps):
        return self.image_shape if smaps is not None else self.maps_shape

    def forward(self, x, smaps=None, out=None, stream=None, reference=False):
        """y[C, M] = A x (unnormalized NUFFT of x*S_c, or of coil images when smaps is None).
        reference=True applies the FP32-class operator of a plan built with
        reference_steps=True (the reference's forward_reference)."""
        torch = _torch()
        cf = torch.complex64
        xp = _dev_ptr(x, cf, self._image_shape(smaps), "x")
        sp = None if smaps is None else _dev_ptr(smaps, cf, self.maps_shape, "smaps")
        if out is None:
            out = torch.empty((self.coils, self.samples), dtype=cf, device=x.device)
        yp = _dev_ptr(out, cf, (self.coils, self.samples), "out")
        fn = lib().tsn_forward_reference if reference else lib().tsn_forward
        check(fn(self._h, xp, sp, yp, _stream_handle(stream)))
        return out

    def adjoint(self, y, smaps=None, out=None, stream=None, reference=False):
        """x = A^H y: coil-combined image [N, N] with smaps, else coil images [C, N, N].
        reference=True: the FP32-class operator (the reference's adjoint_reference)."""
        torch = _torch()
        cf = torch.complex64
        yp = _dev_ptr(y, cf, (self.coils, self.samples), "y")
        sp = None if smaps is None else _dev_ptr(smaps, cf, self.maps_shape, "smaps")
        if out is None:
            out = torch.empty(self._image_shape(smaps), dtype=cf, device=y.device)
        xp = _dev_ptr(out, cf, self._image_shape(smaps), "out")
        fn = lib().tsn_adjoint_reference if reference else lib().tsn_adjoint
        check(fn(self._h, yp, sp, xp, _stream_handle(stream)))
        return out

    def normal(self, p, smaps, *, density=None, lam=0.0, out=None, coils=False, pq=False, p_norm_parts=None,
               stream=None):
        """q = A^H W A p + lam p (tsn_normal): the CG's normal operator on image p [N, N] with
        coil maps.  coils=True also returns the coil images A_c^H W A p [C, N, N] before the
        combine; pq=True also returns Re <p, q> as a 0-d FP64 tensor on the device (no sync).
        p_norm_parts: an FP64 device tensor whose sum is |p|^2 (as cg_step returns for its p'),
        which saves the pass that computes it.
        Returns (q, coil images or None, Re <p, q> or None)."""
        torch = _torch()
        cf = torch.complex64
        pp = _dev_ptr(p, cf, self.image_shape, "p")
        sp = _dev_ptr(smaps, cf, self.maps_shape, "smaps")
        dp = None if density is None else _dev_ptr(density, torch.float32, (self.samples,), "density")
        if out is None:
            out = torch.empty(self.image_shape, dtype=cf, device=p.device)
        qp = _dev_ptr(out, cf, self.image_shape, "out")
        t = torch.empty(self.maps_shape, dtype=cf, device=p.device) if coils else None
        tp = None if t is None else _dev_ptr(t, cf, self.maps_shape, "coils")
        d = torch.empty((), dtype=torch.float64, device=p.device) if pq else None
        if p_norm_parts is not None:
            if p_norm_parts.dtype != torch.float64 or not p_norm_parts.is_cuda or not p_norm_parts.is_contiguous():
                raise TypeError("p_norm_parts must be a contiguous float64 CUDA tensor")
            npp, npn = C.c_void_p(p_norm_parts.data_ptr()), int(p_norm_parts.numel())
        else:
            npp, npn = None, 0
        check(lib().tsn_normal(self._h, pp, sp, dp, float(lam), qp, tp, None if d is None else d.data_ptr(), npp, npn,
                               _stream_handle(stream)))
        return out, t, d

    def rdot(self, a, b, stream=None):
        """Re <a, b> over two complex64 device tensors of one size, FP64 in a fixed order
        (tsn_rdot): a 0-d FP64 tensor on the device (no sync)."""
        torch = _torch()
        if a.numel() != b.numel():
            raise ValueError("rdot needs two tensors of one size")
        ap = _dev_ptr(a, torch.complex64, tuple(a.shape), "a")
        bp = _dev_ptr(b, torch.complex64, tuple(b.shape), "b")
        d = torch.empty((), dtype=torch.float64, device=a.device)
        check(lib().tsn_rdot(self._h, ap, bp, int(a.numel()), d.data_ptr(), _stream_handle(stream)))
        return d

    def cg_step(self, rho, gamma, x, p, r, q, norm_parts=False, stream=None):
        """One CG step on image vectors (tsn_cg_step): returns (x' or None, r', p', rho' as a
        0-d FP64 device tensor, and with norm_parts=True the FP64 partials of |p'|^2 for the
        next normal()) with alpha = rho / gamma; x may be None."""
        torch = _torch()
        shape = tuple(p.shape)
        cf = torch.complex64
        sc = [_dev_ptr(rho, torch.float64, (), "rho"), _dev_ptr(gamma, torch.float64, (), "gamma")]
        xo = None if x is None else torch.empty(shape, dtype=cf, device=p.device)
        ro, po = torch.empty(shape, dtype=cf, device=p.device), torch.empty(shape, dtype=cf, device=p.device)
        rho_o = torch.empty((), dtype=torch.float64, device=p.device)
        parts = torch.empty(_lib.CG_STEP_PARTS, dtype=torch.float64, device=p.device) if norm_parts else None
        check(lib().tsn_cg_step(self._h, int(p.numel()), *sc, None if x is None else _dev_ptr(x, cf, shape, "x"),
                                _dev_ptr(p, cf, shape, "p"), _dev_ptr(r, cf, shape, "r"), _dev_ptr(q, cf, shape, "q"),
                                None if xo is None else C.c_void_p(xo.data_ptr()), C.c_void_p(ro.data_ptr()),
                                C.c_void_p(po.data_ptr()), C.c_void_p(rho_o.data_ptr()),
                                None if parts is None else C.c_void_p(parts.data_ptr()), _stream_handle(stream)))
        return (xo, ro, po, rho_o, parts) if norm_parts else (xo, ro, po, rho_o)

    def cg_adjoint_step(self, rho, rho_next, gamma, rhob, rb, pb, p, q, r_next, xb, norm_parts=False, stream=None):
        """One reverse-mode CG step (tsn_cg_adjoint_step): rb and pb (complex64, one image each)
        are updated in place; returns (qb, the cotangent of rho as a 0-d FP64 device tensor, and
        with norm_parts=True the FP64 partials of |qb|^2 for normal(qb)).
        rho, rho_next, gamma, rhob are 0-d FP64 device tensors."""
        torch = _torch()
        shape = tuple(p.shape)
        ptrs = [_dev_ptr(v, torch.float64, (), nm) for v, nm in
                ((rho, "rho"), (rho_next, "rho_next"), (gamma, "gamma"), (rhob, "rhob"))]
        vec = [_dev_ptr(v, torch.complex64, shape, nm) for v, nm in
               ((rb, "rb"), (pb, "pb"), (p, "p"), (q, "q"), (r_next, "r_next"), (xb, "xb"))]
        qb = torch.empty(shape, dtype=torch.complex64, device=p.device)
        rhob_out = torch.empty((), dtype=torch.float64, device=p.device)
        parts = torch.empty(_lib.CG_STEP_PARTS, dtype=torch.float64, device=p.device) if norm_parts else None
        check(lib().tsn_cg_adjoint_step(self._h, int(p.numel()), *ptrs, C.c_void_p(rhob_out.data_ptr()), *vec,
                                        C.c_void_p(qb.data_ptr()), None if parts is None else C.c_void_p(parts.data_ptr()),
                                        _stream_handle(stream)))
        return (qb, rhob_out, parts) if norm_parts else (qb, rhob_out)

    def cg_adjoint_finish(self, pb, mqb, qb=None, t=None, tb=None, p=None, sb=None, stream=None):
        """pb += mqb in place and, with sb given, sb[c] += conj(qb) t[c] + tb[c] conj(p)
        (tsn_cg_adjoint_finish)."""
        torch = _torch()
        shape = tuple(pb.shape)
        cf = torch.complex64
        args = [_dev_ptr(pb, cf, shape, "pb"), _dev_ptr(mqb, cf, shape, "mqb")]
        if sb is None:
            args += [None, None, None, None, None]
            coils = 0
        else:
            cshape = tuple(sb.shape)
            coils = cshape[0]
            args += [_dev_ptr(qb, cf, shape, "qb"), _dev_ptr(t, cf, cshape, "t"), _dev_ptr(tb, cf, cshape, "tb"),
                     _dev_ptr(p, cf, shape, "p"), _dev_ptr(sb, cf, cshape, "sb")]
        check(lib().tsn_cg_adjoint_finish(self._h, int(pb.numel()), int(coils), *args, _stream_handle(stream)))

    def cg_sense(self, y, smaps, *, density=None, lam=1e-4, iters=10, operator_scale=1.0, out=None, stream=None,
                 sync=True, reliable_update_period=0, reliable_update_direction="restart",
                 scheduled_reference_period=0, reference_steps=()):
        """CG-SENSE solve of (A^H W A + lam) x = A^H W y from x0 = 0 (one CUDA graph).

        Returns (x, residual history or None, status dict or None).  With sync=False
        the call is fully asynchronous and no host-side status is produced.  A positive
        reliable_update_period replaces the recursive residual by b - M x after every that
        many iterations, with p restarted ("restart") or continued ("beta").  On a plan built
        with reference_steps=True, completed iterations that are multiples of
        scheduled_reference_period, or listed in reference_steps (1-based, <= 64), apply the
        normal operator through the FP32-class coefficients (reference_sparse_solver.py cg_sense,
        scheduled_reference_period / explicit_reference_steps).
        """
        torch = _torch()
        cf = torch.complex64
        yp = _dev_ptr(y, cf, (self.coils, self.samples), "y")
        sp = _dev_ptr(smaps, cf, self.maps_shape, "smaps")
        dp = None if density is None else _dev_ptr(density, torch.float32, (self.samples,), "density")
        if out is None:
            out = torch.empty(self.image_shape, dtype=cf, device=y.device)
        xp = _dev_ptr(out, cf, self.image_shape, "out")
        hist = np.zeros(iters + 1, dtype=np.float64) if sync else None
        st = CgStatus() if sync else None
        if reliable_update_direction not in ("restart", "beta"):
            raise ValueError("reliable_update_direction must be 'restart' or 'beta'")
        opts = _lib.CgOptions()
        opts.reliable_update_period = int(reliable_update_period)
        opts.reliable_update_direction = 0 if reliable_update_direction == "restart" else 1
        opts.scheduled_reference_period = int(scheduled_reference_period)
        mask = 0
        for step in reference_steps:
            if not 1 <= int(step) <= 64:
                raise ValueError("reference steps are completed iterations 1..64")
            mask |= 1 << (int(step) - 1)
        opts.reference_steps = mask
        rc = lib().tsn_cg_sense_ex(self._h, yp, sp, dp, float(lam), float(operator_scale), int(iters),
                                   C.byref(opts), xp, ptr(hist, C.c_double), C.byref(st) if sync else None,
                                   _stream_handle(stream))
        status = None
        if sync:
            status = {"completed_iterations": st.completed_iterations,
                      "positive_curvature": bool(st.positive_curvature), "finite": bool(st.finite),
                      "timeout": bool(st.timeout), "residual0": st.residual0, "residual_final": st.residual_final}
            if rc in (4, 5):  # NONFINITE / CURVATURE: reported in the status, x returned as computed
                status["failure"] = _lib.STATUS[rc]
                return out, hist, status
        check(rc)
        return out, hist, status

    def profile_stages(self, y, smaps, reps=20, stream=None) -> dict:
        """Mean milliseconds per launch of each CG-iteration stage (CUDA events)."""
        torch = _torch()
        yp = _dev_ptr(y, torch.complex64, (self.coils, self.samples), "y")
        sp = _dev_ptr(smaps, torch.complex64, self.maps_shape, "smaps")
        out = np.zeros(len(_lib.STAGES), dtype=np.float64)
        check(lib().tsn_profile_stages(self._h, yp, sp, int(reps), ptr(out, C.c_double), _stream_handle(stream)))
        stages = dict(zip(_lib.STAGES, out.tolist()))
        if self.dims == 2:  # images have no middle-axis stages
            stages.pop("fwd_mid")
            stages.pop("inv_mid")
        return stages

    def fft_forward_panel(self, x, smaps=None, stream=None):
        """Forward FFT endpoint: (panel [G*G, 4C] f16 in q1-major rows, panel scale)."""
        torch = _torch()
        xp = _dev_ptr(x, torch.complex64, self._image_shape(smaps), "x")
        sp = None if smaps is None else _dev_ptr(smaps, torch.complex64, self.maps_shape,
                                                 "smaps")
        panel = torch.empty((self.grid_cells, 4 * self.coils), dtype=torch.float16, device=x.device)
        scale = C.c_float(0.0)
        check(lib().tsn_fft_forward_panel(self._h, xp, sp, C.c_void_p(panel.data_ptr()), C.byref(scale),
                                          _stream_handle(stream)))
        return panel, scale.value

    def fft_adjoint_image(self, grid, smaps=None, out=None, stream=None):
        """Adjoint FFT endpoint from a grid [G*G, C] c64 in q1-major rows."""
        torch = _torch()
        gp = _dev_ptr(grid, torch.complex64, (self.grid_cells, self.coils), "grid")
        sp = None if smaps is None else _dev_ptr(smaps, torch.complex64, self.maps_shape,
                                                 "smaps")
        if out is None:
            out = torch.empty(self._image_shape(smaps), dtype=torch.complex64, device=grid.device)
        xp = _dev_ptr(out, torch.complex64, self._image_shape(smaps), "out")
        check(lib().tsn_fft_adjoint_image(self._h, gp, sp, xp, _stream_handle(stream)))
        return out

    def interp_component(self, view: str, component: int, dense_f16):
        """Raw out[rows,16] f32 = component(view) @ dense[n_cols,16] (reference.bin contract)."""
        torch = _torch()
        rows = self.grid_cells if view == "G_T" else self.samples
        cols = self.samples if view == "G_T" else self.grid_cells
        dp = _dev_ptr(dense_f16, torch.float16, (cols, 16), "dense")
        out = torch.zeros((rows, 16), dtype=torch.float32, device=dense_f16.device)
        check(lib().tsn_interp_component(self._h, _lib.VIEW[view], int(component), dp, C.c_void_p(out.data_ptr()),
                                         _stream_handle(None)))
        return out


class Batch:
    """Independent plans solved together (tsn_batch_*): one CUDA graph forks the cases over
    `streams` streams and each case's persistent launches use a 1/streams slice of the GPU.

    The plans stay owned by the caller and must outlive the batch."""

    def __init__(self, plans, streams: int = 0):
        self.plans = list(plans)
        if not self.plans:
            raise ValueError("a batch needs at least one plan")
        arr = (C.c_void_p * len(self.plans))(*[pl._h.value for pl in self.plans])
        h = C.c_void_p()
        check(lib().tsn_batch_create(arr, len(self.plans), int(streams), C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().tsn_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def cg_sense(self, ys, smaps, *, densities=None, lam=1e-4, iters=10, operator_scale=1.0, outs=None,
                 stream=None, sync=True):
        """CG-SENSE of every case; returns (list of x, list of status dicts or None).

        A case whose solve went non-finite or lost positive curvature is reported in its
        status (key "failure"); its x is returned as computed."""
        torch = _torch()
        cf = torch.complex64
        n_cases = len(self.plans)
        if len(ys) != n_cases or len(smaps) != n_cases:
            raise ValueError("one y and one smaps per case")
        if outs is None:
            outs = [torch.empty(pl.image_shape, dtype=cf, device=y.device) for pl, y in zip(self.plans, ys)]
        yp, sp, dp, xp = [], [], [], []
        for i, pl in enumerate(self.plans):
            yp.append(_dev_ptr(ys[i], cf, (pl.coils, pl.samples), f"ys[{i}]").value)
            sp.append(_dev_ptr(smaps[i], cf, pl.maps_shape, f"smaps[{i}]").value)
            w = None if densities is None else densities[i]
            dp.append(None if w is None else _dev_ptr(w, torch.float32, (pl.samples,), f"densities[{i}]").value)
            xp.append(_dev_ptr(outs[i], cf, pl.image_shape, f"outs[{i}]").value)
        arr = lambda v: (C.c_void_p * n_cases)(*v)
        st = (CgStatus * n_cases)() if sync else None
        rc = lib().tsn_batch_cg_sense(self._h, arr(yp), arr(sp), arr(dp), float(lam), float(operator_scale),
                                      int(iters), arr(xp), st, _stream_handle(stream))
        statuses = None
        if sync:
            statuses = []
            for s_ in st:
                d = {"completed_iterations": s_.completed_iterations,
                     "positive_curvature": bool(s_.positive_curvature), "finite": bool(s_.finite),
                     "timeout": bool(s_.timeout), "residual0": s_.residual0, "residual_final": s_.residual_final}
                if not d["finite"]:
                    d["failure"] = "NONFINITE"
                elif not d["positive_curvature"]:
                    d["failure"] = "CURVATURE"
                statuses.append(d)
            if rc in (4, 5):
                return outs, statuses
        check(rc)
        return outs, statuses


def load_runtime_dir(directory, coils: int, im_size: int, samples: int) -> dict:
    """Runtime inputs in the reference layout (export_real_runtime_inputs.py:97-113)."""
    d = Path(directory)
    out = {
        "measurement": np.fromfile(d / "measurement.c64.bin", dtype=np.complex64).reshape(coils, samples),
        "sensitivity_maps": np.fromfile(d / "sensitivity_maps.c64.bin", dtype=np.complex64).reshape(
            coils, im_size, im_size),
        "scaling": np.fromfile(d / "scaling.f32.bin", dtype=np.float32).reshape(im_size, im_size),
    }
    if (d / "density.f32.bin").exists():
        out["density"] = np.fromfile(d / "density.f32.bin", dtype=np.float32).reshape(samples)
    return out


def write_runtime_dir(directory, measurement, sensitivity_maps, scaling, density=None, truth=None) -> Path:
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    np.ascontiguousarray(measurement, dtype=np.complex64).tofile(d / "measurement.c64.bin")
    np.ascontiguousarray(sensitivity_maps, dtype=np.complex64).tofile(d / "sensitivity_maps.c64.bin")
    np.ascontiguousarray(scaling, dtype=np.float32).tofile(d / "scaling.f32.bin")
    if density is not None:
        np.ascontiguousarray(density, dtype=np.float32).tofile(d / "density.f32.bin")
    if truth is not None:
        np.ascontiguousarray(truth, dtype=np.complex64).tofile(d / "truth.c64.bin")
    return d
