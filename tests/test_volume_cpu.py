"""Volume (3D kooshball) pieces that need no GPU: the C++ KB weights and deapodization
against the oracle, the FP64 3D NUDFT against a brute-force sum, the FP64 KB operator
against the NUDFT, and the synthetic kooshball trajectory."""
import math

import numpy as np
import pytest

from oracle import kb as okb
from oracle import nudft as onudft
from oracle import operator as oop
from trajsparsenufft_b200 import synth


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def test_kooshball_trajectory():
    t = synth.kooshball(128, 32).astype(np.float64)
    assert t.shape == (128 * 32, 3) and np.all(np.abs(t) <= 0.5)
    spokes = t.reshape(128, 32, 3)
    # sample 0 of a spoke is radius -0.5 along its unit direction
    assert np.allclose(np.linalg.norm(spokes[:, 0], axis=-1), 0.5, atol=1e-6)
    p1, p2 = synth.GOLDEN_MEANS_3D
    assert abs(p2 ** 3 + p2 - 1.0) < 1e-14 and abs(p1 - p2 * p2) < 1e-14


def test_library_kb_weights_match_oracle():
    from trajsparsenufft_b200 import packing
    traj = synth.kooshball(64, 32)
    rp, cols, w = packing.kb_weights_csr3(traj, 16, 32, 4)
    orp, ocols, ow = okb.weights_csr3(traj, 16, 32, 4)
    assert np.array_equal(rp, orp) and np.array_equal(cols, ocols)
    assert np.max(np.abs(w - ow)) <= 1e-14 * np.max(ow)
    d = packing.kb_deapodization3(16, 32, 4)
    assert np.max(np.abs(d / okb.deapodization3(16, 32, 4) - 1.0)) <= 1e-14


def test_nudft3_matches_brute_force():
    n, c = 8, 2
    traj = synth.kooshball(8, 8)
    rng = np.random.default_rng(3)
    x = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    s = rng.standard_normal((c, n, n, n)) + 1j * rng.standard_normal((c, n, n, n))
    y = onudft.Nudft3(traj, n).forward(x, s)
    i = np.arange(n) - n // 2
    grid = np.stack(np.meshgrid(i, i, i, indexing="ij"), axis=-1).astype(np.float64)
    w = 2.0 * math.pi * traj.astype(np.float64)
    brute = np.stack([np.sum(x[None] * s * np.exp(-1j * (grid @ w[m]))[None], axis=(1, 2, 3))
                      for m in range(len(traj))], axis=1)
    assert _rel(y, brute) <= 1e-12
    yr = rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape)
    a = onudft.Nudft3(traj, n).adjoint(yr, s)
    assert abs(np.vdot(yr, y) - np.vdot(a, x)) <= 1e-11 * np.linalg.norm(yr) * np.linalg.norm(y)


def test_kb_operator3_close_to_nudft3_and_adjoint():
    n, g, c = 16, 32, 3
    traj = synth.kooshball(48, 32)
    x = synth.ellipsoid_phantom(n, 5)
    s = synth.coil_maps3(n, c, 5)
    exact = onudft.Nudft3(traj, n)
    y = exact.forward(x, s)
    op6 = oop.KbSenseOperator3(traj, n, g, 6)
    op4 = oop.KbSenseOperator3(traj, n, g, 4)
    assert _rel(op6.forward(x, s), y) <= 2e-5
    assert _rel(op4.forward(x, s), y) <= 3e-3
    rng = np.random.default_rng(7)
    yr = rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape)
    assert _rel(op6.adjoint(yr, s), exact.adjoint(yr, s)) <= 2e-5
    yk = op4.forward(x, s)
    ak = op4.adjoint(yr, s)
    assert abs(np.vdot(yr, yk) - np.vdot(ak, x.astype(np.complex128))) <= 1e-12 * np.linalg.norm(yr) * np.linalg.norm(yk)


@pytest.mark.parametrize("n", [16, 24])
def test_volume_phantom_and_maps(n):
    x = synth.ellipsoid_phantom(n, 9)
    s = synth.coil_maps3(n, 8, 9)
    assert x.shape == (n, n, n) and x.dtype == np.complex64 and np.abs(x).max() > 0.1
    assert s.shape == (8, n, n, n)
    assert np.allclose(np.sqrt(np.sum(np.abs(s) ** 2, axis=0)), 1.0, atol=1e-5)


@pytest.mark.parametrize("kw,kind", [
    (dict(grid_size=512, im_size=256), "UNSUPPORTED"),          # 512^3 cells > 2^24 record rows
    (dict(reference_layout=True), "UNSUPPORTED"),              # volumes use the centred layout
])
def test_volume_plan_refusals_before_any_device_work(kw, kind):
    """Volume plans that the library cannot serve are refused with a status before any CUDA
    call, so these run without a GPU."""
    from trajsparsenufft_b200._lib import TsnError
    from trajsparsenufft_b200.operator import Plan
    args = dict(im_size=64, grid_size=128, coils=4, width=4, device=0)
    args.update(kw)
    with pytest.raises(TsnError) as e:
        Plan.from_trajectory(synth.kooshball(8, 16), **args)
    assert e.value.kind == kind


def test_volume_trajectory_and_dims_validation():
    from trajsparsenufft_b200 import _lib
    from trajsparsenufft_b200._lib import TsnError
    from trajsparsenufft_b200.operator import Plan, plan_desc
    bad = synth.kooshball(8, 16) * 1.5                          # outside [-0.5, 0.5]
    with pytest.raises(TsnError) as e:
        Plan.from_trajectory(bad, im_size=64, grid_size=128, coils=4, width=4, device=0)
    assert e.value.kind == "ARG"
    d = plan_desc(64, 128, 4, 4, dims=4, device=0)
    t = np.ascontiguousarray(synth.kooshball(8, 16))
    import ctypes as C
    h = C.c_void_p()
    rc = _lib.lib().tsn_plan_create_from_trajectory(t.ctypes.data_as(C.POINTER(C.c_float)), len(t), C.byref(d),
                                                    C.byref(h))
    assert _lib.STATUS[rc] == "ARG" and not h.value


def test_pack_directories_are_refused_for_volumes():
    import ctypes as C
    from trajsparsenufft_b200 import _lib
    from trajsparsenufft_b200.operator import plan_desc
    d = plan_desc(64, 128, 4, 4, dims=3, device=0)
    h = C.c_void_p()
    rc = _lib.lib().tsn_plan_create_from_pack(b"/nonexistent/r", b"/nonexistent/i", None, None, None, C.byref(d),
                                              C.byref(h))
    assert _lib.STATUS[rc] == "UNSUPPORTED" and not h.value
