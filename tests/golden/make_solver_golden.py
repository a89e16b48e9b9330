#!/usr/bin/env python3
"""Generate the reference-solver fixture by running the reference's own CG-SENSE code.

    python tests/golden/make_solver_golden.py --reference-root <path of the reference checkout>

(or set TSN_REFERENCE_ROOT).  The GPU box never runs this script; tests read only the file it
writes next to it (solver_small.npz).

What runs
---------
experiments/production/reference_sparse_solver.py, imported unchanged:
``make_component_operator`` (:131-197) with ``sparse_layout="csr"`` on the CPU, then
``cg_sense`` (:200-332), for two arithmetic variants of its VARIANTS table (:37-45):

* ``fp32x32``: matrix "fp32", panel "fp32" (the FP32 CPU path that bench.py's CPU baseline
  restates in oracle/cpu_ref.py);
* ``fp16x2``: matrix "fp16", panel "split2" (the FP16 high + FP16 residual arithmetic of
  the GPU path, restated in oracle/operator.py).

Two imports of that module are absent here and are stubbed in ``sys.modules``:

* ``torchkbnufft`` 1.5.2 (requirements-gpu.txt:5).  The solver calls only its
  ``_nufft.fft.fft_and_scale`` / ``ifft_and_scale`` (:157-163, :188-194).  The stubs restate
  what those do with ``norm=None``: multiply by the scaling coefficients, zero-pad each image
  axis at its end to the grid size and take the unnormalized FFT; and the exact adjoint of
  that (unnormalized inverse FFT, crop to the image size, multiply by the conjugated
  scaling coefficients).  The solver's ``forward_op`` / ``adjoint_op`` arguments are plain
  objects carrying ``scaling_coef``, ``im_size`` and ``grid_size``.
* ``skimage.metrics`` (used by the module's CLI only, never by the two functions above).

Inputs (all seeded): a 64 x 64 random-ellipse phantom, 4 Gaussian-blob coil maps,
golden-angle radial 32 spokes x 128 samples, grid 128, KB width 6 coefficients from
oracle/kb.py (the reference's coefficients come from torchkbnufft, which is absent), the
[0, N) deapodization table of oracle/kb.py, k-space = FP64 direct NUDFT + 1e-3 rms noise,
lambda 1e-4, 10 iterations.  The fp16x2 run solves the same system rescaled by powers of two
(maps x 2^fp16x2_maps_scale_exp, lambda x 2^(2 fp16x2_maps_scale_exp), data x
2^fp16x2_data_scale_exp, all stored), which keeps its FP16 panels in range.
"""

from __future__ import annotations

import argparse
import importlib
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from oracle import kb, nudft  # noqa: E402
from trajsparsenufft_b200 import synth  # noqa: E402

N, G, C, J, SPOKES, READOUT, ITERS, LAM = 64, 128, 4, 6, 32, 128, 10, 1e-4
SEED = synth.BASE_SEED


def _stub_modules(torch) -> None:
    """torchkbnufft FFT helpers and skimage.metrics stand-ins (see the module docstring)."""

    def fft_and_scale(image, scaling_coef, im_size, grid_size, norm=None):
        assert norm is None
        n = [int(v) for v in im_size]
        g = [int(v) for v in grid_size]
        scaled = image * scaling_coef
        padded = torch.zeros(scaled.shape[:-2] + tuple(g), dtype=scaled.dtype)
        padded[..., : n[0], : n[1]] = scaled
        return torch.fft.fftn(padded, dim=(-2, -1))

    def ifft_and_scale(image, scaling_coef, im_size, grid_size, norm=None):
        assert norm is None
        n = [int(v) for v in im_size]
        g = [int(v) for v in grid_size]
        full = torch.fft.ifftn(image, dim=(-2, -1)) * float(g[0] * g[1])
        return full[..., : n[0], : n[1]] * scaling_coef.conj()

    tkbn = types.ModuleType("torchkbnufft")
    nufft = types.ModuleType("torchkbnufft._nufft")
    fft = types.ModuleType("torchkbnufft._nufft.fft")
    fft.fft_and_scale = fft_and_scale
    fft.ifft_and_scale = ifft_and_scale
    nufft.fft = fft
    tkbn._nufft = nufft
    sys.modules["torchkbnufft"] = tkbn
    sys.modules["torchkbnufft._nufft"] = nufft
    sys.modules["torchkbnufft._nufft.fft"] = fft

    def _cli_only(*_a, **_k):
        raise RuntimeError("skimage.metrics is used by the reference CLI only")

    skimage = types.ModuleType("skimage")
    metrics = types.ModuleType("skimage.metrics")
    metrics.peak_signal_noise_ratio = _cli_only
    metrics.structural_similarity = _cli_only
    skimage.metrics = metrics
    sys.modules["skimage"] = skimage
    sys.modules["skimage.metrics"] = metrics


def inputs():
    """The fixture's seeded inputs (also rebuilt by the tests from the same seeds)."""
    traj = synth.golden_radial(SPOKES, READOUT)
    x = synth.ellipse_phantom(N, SEED)
    s = synth.coil_maps(N, C, SEED)
    y = synth.add_noise(nudft.Nudft(traj, N).forward(x, s), SEED).astype(np.complex64)
    return traj, x, s, y


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference-root", default=os.environ.get("TSN_REFERENCE_ROOT"),
                    help="root of the reference checkout (or TSN_REFERENCE_ROOT)")
    args = ap.parse_args()
    if not args.reference_root:
        ap.error("name the reference checkout with --reference-root or TSN_REFERENCE_ROOT")
    root = Path(args.reference_root)
    src = root / "experiments" / "production" / "reference_sparse_solver.py"
    if not src.is_file():
        print(f"reference solver not found under {root}", file=sys.stderr)
        return 2
    import torch

    torch.manual_seed(0)
    _stub_modules(torch)
    sys.path.insert(0, str(src.parent))
    ref = importlib.import_module("reference_sparse_solver")

    traj, x, s, y = inputs()
    row_ptr, cols, re, im = kb.interpolation_csr(traj, N, G, J)
    m = len(row_ptr) - 1
    rows = np.repeat(np.arange(m), np.diff(row_ptr))
    idx = torch.from_numpy(np.stack([rows, cols]).astype(np.int64))
    real_m = torch.sparse_coo_tensor(idx, torch.from_numpy(re), (m, G * G))
    imag_m = torch.sparse_coo_tensor(idx, torch.from_numpy(im), (m, G * G))
    scaling = torch.from_numpy(kb.deapodization(N, G, J).astype(np.float32)).to(torch.complex64)
    op = types.SimpleNamespace(scaling_coef=scaling, im_size=torch.tensor([N, N]), grid_size=torch.tensor([G, G]))
    smaps = torch.from_numpy(s.astype(np.complex64)).unsqueeze(0)
    data = torch.from_numpy(y).unsqueeze(0)
    out = {"trajectory": traj, "image": x.astype(np.complex64), "smaps": s.astype(np.complex64), "data": y,
           "kb_checksum": np.array([re.sum(), im.sum(), np.abs(re).sum(), float(cols.sum())]),
           "shape": np.array([N, G, C, J, ITERS]), "lam": np.float64(LAM)}
    # The fp16x2 variant splits its panels into FP16 without any scaling.  In these raw NUFFT
    # units the forward panel (the FFT of the CG iterate, which starts at A^H y) is ~10^5 times
    # larger than the sample panel, so one of them always falls into FP16 subnormals or
    # overflows (the reference CUDA passes an operator scale and divides its measurement by
    # the grid size for this, nufft_fp16x2_cg_bench.cu:330-334, :401-404).  That variant
    # therefore runs on an exactly rescaled system: maps x 2^a, lambda x 2^(2a), data x 2^k
    # (powers of two, exact in every precision involved), whose solution is x 2^(k - a) and
    # whose residuals are scaled by 2^(a + k); a balances the two panels, k puts them near 2^10.
    fwd32, adj32 = ref.make_component_operator(op, op, real_m, imag_m, smaps, "fp32", "fp32", C, G,
                                               torch.device("cpu"), "csr")
    b = adj32(data)
    peak_grid = float(torch.fft.fftn(b * smaps * scaling, s=(G, G), dim=(-2, -1)).abs().max())
    peak_data = float(data.abs().max())
    a_exp = int(np.round(0.5 * np.log2(peak_data / peak_grid)))
    k_exp = int(np.floor(np.log2(2.0 ** 10 / max(peak_data, peak_grid * 2.0 ** (2 * a_exp)))))
    out["fp16x2_maps_scale_exp"] = np.int64(a_exp)
    out["fp16x2_data_scale_exp"] = np.int64(k_exp)
    for tag, (matrix_mode, panel_mode) in (("fp32x32", ("fp32", "fp32")), ("fp16x2", ("fp16", "split2"))):
        scaled = tag == "fp16x2"
        run_maps = smaps * (2.0 ** a_exp) if scaled else smaps
        run_data = data * (2.0 ** k_exp) if scaled else data
        run_lam = LAM * (2.0 ** (2 * a_exp)) if scaled else LAM
        fwd, adj = ref.make_component_operator(op, op, real_m, imag_m, run_maps, matrix_mode, panel_mode, C, G,
                                               torch.device("cpu"), "csr")
        xr, residuals, status = ref.cg_sense(fwd, adj, run_data, ITERS, run_lam, tag, False)
        assert status["finite"] and status["positive_curvature"] and status["completed_iterations"] == ITERS
        out[f"x_{tag}"] = xr.squeeze().numpy().astype(np.complex64)
        out[f"residuals_{tag}"] = np.asarray(residuals, dtype=np.float64)
        out[f"denominators_{tag}"] = np.asarray([b["denominator"] for b in status["curvature_history"]])
        # one forward / adjoint application of the variant, for operator-level checks
        xin = torch.from_numpy(x.astype(np.complex64))[None, None]
        if scaled:  # an image of the magnitude of the rescaled right-hand side 2^(a + k) A^H y
            xin = xin * float(2.0 ** round(np.log2(np.abs(b.numpy()).max() / np.abs(x).max())) * 2.0 ** (k_exp + a_exp))
        out[f"forward_input_{tag}"] = xin.squeeze().numpy()
        out[f"forward_{tag}"] = fwd(xin).squeeze(0).numpy()
        out[f"adjoint_{tag}"] = adj(run_data).squeeze().numpy()
    np.savez_compressed(HERE / "solver_small.npz", **out)
    print(f"wrote {HERE / 'solver_small.npz'}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
