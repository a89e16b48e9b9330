"""Volume (3D kooshball) plans on the GPU against the oracle (marked gpu).

Tolerances (written here):
* forward / adjoint vs the FP64 KB operator with FP16 weights and FP16 high + residual
  panels emulated (the same arithmetic): rel_l2 <= 2e-5;
* vs the FP64 KB operator with J = 6 (within 1e-5 of the direct NUDFT at these sizes) and
  vs the direct FP64 NUDFT on a 768-sample subsample: rel_l2 <= 3e-3 (the KB J = 4
  approximation error of the 3D configuration, ~1e-3);
* FFT endpoints vs numpy fftn / ifftn: rel_l2 <= 1e-5;
* adjointness |<y,Ax> - <A^H y,x>| / (|y| |Ax|) <= 1e-5;
* CG-SENSE reconstruction magnitude NRMSE vs FP64 CG with the same KB operator <= 2e-3.
"""
import numpy as np
import pytest

from gpu_cases import rel_l2, volume_case, volume_measurement
from oracle import kb as okb
from oracle import nudft as onudft
from oracle import operator as oop
from trajsparsenufft_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _plan(name, **kw):
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j = volume_case(name)
    return Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j, **kw)


def test_volume_plan_info():
    plan = _plan("vol64")
    traj, x, s, n, g, c, j = volume_case("vol64")
    info = plan.info
    assert info["dims"] == 3 and plan.image_shape == (n, n, n) and plan.grid_cells == g ** 3
    assert info["samples"] == len(traj) and info["components"] == 1
    assert info["nnz"][0] == info["nnz"][1] > 0 and min(info["tiles"]) > 0


def test_volume_forward_panel_matches_numpy_fftn():
    plan = _plan("vol64")
    traj, x, s, n, g, c, j = volume_case("vol64")
    panel, scale = plan.fft_forward_panel(torch.from_numpy(x).cuda(), torch.from_numpy(s).cuda())
    p = panel.float().cpu().numpy().astype(np.float64)           # [G^3, 4C], rows (q2*G + q1)*G + q0
    v = (p[:, : 2 * c] + p[:, 2 * c:])
    v = v[:, 0::2] + 1j * v[:, 1::2]
    got = v.reshape(g, g, g, c).transpose(3, 2, 1, 0) / scale     # [C, q0, q1, q2]
    pos = (np.arange(n) - n // 2) % g
    grid = np.zeros((c, g, g, g), dtype=np.complex128)
    grid[np.ix_(np.arange(c), pos, pos, pos)] = x[None] * s * okb.deapodization3(n, g, j)[None]
    assert rel_l2(got, np.fft.fftn(grid, axes=(1, 2, 3))) <= 1e-5


def test_volume_adjoint_endpoint_matches_numpy_ifftn():
    plan = _plan("vol64")
    traj, x, s, n, g, c, j = volume_case("vol64")
    rng = np.random.default_rng(5)
    grid = (rng.standard_normal((c, g, g, g)) + 1j * rng.standard_normal((c, g, g, g))).astype(np.complex64)
    internal = np.ascontiguousarray(grid.transpose(3, 2, 1, 0).reshape(g ** 3, c))
    got = plan.fft_adjoint_image(torch.from_numpy(internal).cuda()).cpu().numpy()       # coil volumes
    pos = (np.arange(n) - n // 2) % g
    full = np.fft.ifftn(grid.astype(np.complex128), axes=(1, 2, 3)) * g ** 3
    want = full[np.ix_(np.arange(c), pos, pos, pos)] * okb.deapodization3(n, g, j)[None]
    assert rel_l2(got, want) <= 1e-5


@pytest.mark.parametrize("name", ["vol64", "vol64c8"])
def test_volume_forward_adjoint_match_oracle(name):
    traj, x, s, n, g, c, j = volume_case(name)
    plan = _plan(name)
    xt, st = torch.from_numpy(x).cuda(), torch.from_numpy(s).cuda()
    y_gpu = plan.forward(xt, st).cpu().numpy()
    emu = oop.KbSenseOperator3(traj, n, g, j, matrix_mode="fp16", panel_mode="split2", workers=8)
    ref6 = oop.KbSenseOperator3(traj, n, g, 6, workers=8)
    assert rel_l2(y_gpu, emu.forward(x, s)) <= 2e-5
    assert rel_l2(y_gpu, ref6.forward(x, s)) <= 3e-3
    sub = np.arange(0, len(traj), max(1, len(traj) // 768))
    exact = onudft.Nudft3(traj[sub], n).forward(x, s)
    assert rel_l2(y_gpu[:, sub], exact) <= 3e-3
    rng = np.random.default_rng(11)
    yr = (rng.standard_normal((c, len(traj))) + 1j * rng.standard_normal((c, len(traj)))).astype(np.complex64)
    a_gpu = plan.adjoint(torch.from_numpy(yr).cuda(), st).cpu().numpy()
    assert rel_l2(a_gpu, emu.adjoint(yr, s)) <= 2e-5
    assert rel_l2(a_gpu, ref6.adjoint(yr, s)) <= 3e-3
    gap = abs(np.vdot(yr.astype(np.complex128), y_gpu) - np.vdot(a_gpu.astype(np.complex128), x))
    assert gap / (np.linalg.norm(yr) * np.linalg.norm(y_gpu)) <= 1e-5
    # coil-volume variants (smaps = NULL)
    coil = (x[None] * s).astype(np.complex64)
    yc = plan.forward(torch.from_numpy(coil).cuda()).cpu().numpy()
    assert rel_l2(yc, y_gpu) <= 1e-5
    ac = plan.adjoint(torch.from_numpy(yr).cuda()).cpu().numpy()
    assert rel_l2(np.sum(np.conj(s) * ac, axis=0), a_gpu) <= 1e-5


def test_volume_cg_sense_matches_oracle():
    traj, x, s, n, g, c, j = volume_case("vol64")
    plan = _plan("vol64")
    y = volume_measurement("vol64")
    xg, hist, status = plan.cg_sense(torch.from_numpy(y).cuda(), torch.from_numpy(s).cuda(), lam=1e-4, iters=10)
    assert status["positive_curvature"] and status["finite"] and status["completed_iterations"] == 10
    assert hist[-1] < 0.5 * hist[0]
    op = oop.KbSenseOperator3(traj, n, g, j, workers=8)
    xo, ho, so = oop.cg_sense(lambda v: op.forward(v, s), lambda v: op.adjoint(v, s), y, 10, 1e-4)
    assert so["completed_iterations"] == 10
    assert oop.magnitude_nrmse(xg.cpu().numpy(), xo) <= 2e-3
    # normalized residual histories agree to 5e-4 absolute (late residuals are at the noise
    # floor, where FP16x2 arithmetic and FP64 differ by a few percent relative)
    assert np.allclose(np.asarray(hist) / hist[0], np.asarray(ho) / ho[0], rtol=2e-3, atol=5e-4)


def test_volume_and_image_in_one_batch_match_single_solves():
    from trajsparsenufft_b200.operator import Batch, Plan
    from gpu_cases import case, torch_inputs
    vol = _plan("vol64c8")
    traj, x, s, n, g, c, j = volume_case("vol64c8")
    yv = torch.from_numpy(volume_measurement("vol64c8")).cuda()
    sv = torch.from_numpy(s).cuda()
    t2, x2, s2, n2, g2, c2, j2, _ = case("small")
    img = Plan.from_trajectory(t2, im_size=n2, grid_size=g2, coils=c2, width=j2)
    _, st2, y2 = torch_inputs("small")
    single_v, _, _ = vol.cg_sense(yv, sv, lam=1e-4, iters=6)
    single_i, _, _ = img.cg_sense(y2, st2, lam=1e-4, iters=6)
    batch = Batch([vol, img], streams=2)
    outs, statuses = batch.cg_sense([yv, y2], [sv, st2], lam=1e-4, iters=6)
    assert all(s_["finite"] and s_["positive_curvature"] for s_ in statuses)
    assert torch.equal(outs[0], single_v) and torch.equal(outs[1], single_i)


def test_volume_density_and_reliable_update():
    """Density-weighted CG and the reliable-update CG (restart every 4 iterations) on a volume
    plan against FP64 restatements with the same KB operator (W enters A^H W A and A^H W y)."""
    from test_gpu_operator import _oracle_reliable_cg
    traj, x, s, n, g, c, j = volume_case("vol64c8")
    plan = _plan("vol64c8")
    y = volume_measurement("vol64c8")
    w = synth.ramp_density(traj)
    yt, st, wt = torch.from_numpy(y).cuda(), torch.from_numpy(s).cuda(), torch.from_numpy(w).cuda()
    op = oop.KbSenseOperator3(traj, n, g, j, workers=8)
    fwd = lambda v: op.forward(v, s)
    adj = lambda v: op.adjoint(v, s)
    w64 = w.astype(np.float64)
    xo, _ = _oracle_reliable_cg(fwd, adj, y, w64, 10, 1e-4, 0, "restart")
    xg, _, status = plan.cg_sense(yt, st, density=wt, lam=1e-4, iters=10)
    assert status["finite"] and status["positive_curvature"]
    assert oop.magnitude_nrmse(xg.cpu().numpy(), xo) <= 2e-3
    xr_o, res_o = _oracle_reliable_cg(fwd, adj, y, w64, 10, 1e-4, 4, "restart")
    xr, hist, status = plan.cg_sense(yt, st, density=wt, lam=1e-4, iters=10, reliable_update_period=4,
                                     reliable_update_direction="restart")
    assert status["finite"] and status["completed_iterations"] == 10
    assert oop.magnitude_nrmse(xr.cpu().numpy(), xr_o) <= 2e-3
    np.testing.assert_allclose(hist[:4], res_o[:4], rtol=2e-3)


def test_two_volume_batch_on_slices_matches_single_solves():
    from trajsparsenufft_b200.operator import Batch
    a, b = _plan("vol64"), _plan("vol64c8")
    ta, xa, sa, *_ = volume_case("vol64")
    tb, xb, sb, *_ = volume_case("vol64c8")
    ya, yb = torch.from_numpy(volume_measurement("vol64")).cuda(), torch.from_numpy(volume_measurement("vol64c8")).cuda()
    sa_t, sb_t = torch.from_numpy(sa).cuda(), torch.from_numpy(sb).cuda()
    single_a, _, _ = a.cg_sense(ya, sa_t, lam=1e-4, iters=5)
    single_b, _, _ = b.cg_sense(yb, sb_t, lam=1e-4, iters=5)
    outs, statuses = Batch([a, b], streams=2).cg_sense([ya, yb], [sa_t, sb_t], lam=1e-4, iters=5)
    assert all(st_["finite"] for st_ in statuses)
    assert torch.equal(outs[0], single_a) and torch.equal(outs[1], single_b)
