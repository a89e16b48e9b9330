"""The CPU restatements of the reference's CG-SENSE solver, pinned to the reference's own output.

tests/golden/solver_small.npz holds what experiments/production/reference_sparse_solver.py
itself computed (tests/golden/make_solver_golden.py ran ``make_component_operator`` and
``cg_sense`` unchanged, CSR layout, CPU) for two variants:

* fp32x32 (matrix fp32, panel fp32): restated by oracle/cpu_ref.py, the timed CPU baseline;
* fp16x2 (matrix fp16, panel split2): restated by oracle/operator.py, the emulation the GPU
  path is checked against.  The reference ran it on the same system rescaled exactly by powers
  of two (maps x 2^a, lambda x 2^2a, data x 2^k, stored) so that its unscaled FP16 split stays
  in range; the comparisons undo that scaling.

Gates (written here): one operator application <= 1e-6 rel (FP32 rounding order only);
10-iteration CG images <= 2e-4 rel and residual histories rtol 2e-3 (FP32 dot products
accumulated in different orders); the FP64 CG of oracle/operator.py within 1e-4 of the
reference's FP32 CG.
"""
import numpy as np
import pytest

from golden_io import GOLDEN
from oracle import cpu_ref, kb
from oracle import operator as oop
from trajsparsenufft_b200 import synth

FIX = GOLDEN / "solver_small.npz"


def _rel(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def fix():
    d = dict(np.load(FIX))
    n, g, c, j, iters = (int(v) for v in d["shape"])
    d.update(n=n, g=g, c=c, j=j, iters=iters, lam=float(d["lam"]),
             a=int(d["fp16x2_maps_scale_exp"]), k=int(d["fp16x2_data_scale_exp"]))
    return d


def test_fixture_inputs_regenerate_from_seeds(fix):
    """The fixture's inputs are the seeded synthetic ones, so its outputs belong to them."""
    from oracle import nudft
    traj = synth.golden_radial(32, 128)
    np.testing.assert_array_equal(traj, fix["trajectory"])
    np.testing.assert_array_equal(synth.ellipse_phantom(fix["n"], synth.BASE_SEED).astype(np.complex64), fix["image"])
    np.testing.assert_array_equal(synth.coil_maps(fix["n"], fix["c"], synth.BASE_SEED).astype(np.complex64),
                                  fix["smaps"])
    y = synth.add_noise(nudft.Nudft(traj, fix["n"]).forward(fix["image"].astype(np.complex128),
                                                            fix["smaps"].astype(np.complex128)), synth.BASE_SEED)
    assert _rel(y, fix["data"]) < 1e-6
    row_ptr, cols, re, im = kb.interpolation_csr(traj, fix["n"], fix["g"], fix["j"])
    np.testing.assert_allclose([re.sum(), im.sum(), np.abs(re).sum(), float(cols.sum())], fix["kb_checksum"],
                               rtol=1e-12)


def test_cpu_port_matches_reference_fp32_solver(fix):
    op = cpu_ref.CpuSenseFp32(fix["trajectory"], fix["n"], fix["g"], fix["j"], fix["smaps"], threads=4)
    assert _rel(op.forward(fix["forward_input_fp32x32"]), fix["forward_fp32x32"]) <= 1e-6
    assert _rel(op.adjoint(fix["data"]), fix["adjoint_fp32x32"]) <= 1e-6
    x, res, _, _ = op.cg_sense(fix["data"], fix["iters"], fix["lam"])
    assert _rel(x, fix["x_fp32x32"]) <= 2e-4
    np.testing.assert_allclose(res, fix["residuals_fp32x32"], rtol=2e-3)


def test_fp16x2_emulation_matches_reference_fp16x2_solver(fix):
    a, k = fix["a"], fix["k"]
    s = fix["smaps"].astype(np.complex128)
    emu = oop.KbSenseOperator(fix["trajectory"], fix["n"], fix["g"], fix["j"], matrix_mode="fp16",
                              panel_mode="split2")
    # one application of the rescaled operator (the emulation's own power-of-two panel scaling
    # commutes with FP16 rounding, so it agrees with the reference's unscaled split in range)
    s2 = s * 2.0 ** a
    assert _rel(emu.forward(fix["forward_input_fp16x2"], s2), fix["forward_fp16x2"]) <= 1e-6
    assert _rel(emu.adjoint(fix["data"].astype(np.complex128) * 2.0 ** k, s2), fix["adjoint_fp16x2"]) <= 1e-6
    # the CG on the original system against the reference's rescaled solve, scaling undone
    x, res, status = oop.cg_sense(lambda v: emu.forward(v, s), lambda v: emu.adjoint(v, s),
                                  fix["data"].astype(np.complex128), fix["iters"], fix["lam"])
    assert status["completed_iterations"] == fix["iters"]
    assert _rel(x, fix["x_fp16x2"] * 2.0 ** (a - k)) <= 2e-4
    np.testing.assert_allclose(res, fix["residuals_fp16x2"] * 2.0 ** -(a + k), rtol=2e-3)


def test_fp64_oracle_cg_matches_reference_fp32_solver(fix):
    s = fix["smaps"].astype(np.complex128)
    op = oop.KbSenseOperator(fix["trajectory"], fix["n"], fix["g"], fix["j"])
    x, res, _ = oop.cg_sense(lambda v: op.forward(v, s), lambda v: op.adjoint(v, s),
                             fix["data"].astype(np.complex128), fix["iters"], fix["lam"])
    assert _rel(x, fix["x_fp32x32"]) <= 1e-4
    np.testing.assert_allclose(res, fix["residuals_fp32x32"], rtol=2e-3)
