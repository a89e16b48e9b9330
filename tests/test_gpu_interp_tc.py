"""The tcgen05.mma.sp interpolation (TSN_INTERP_TCGEN05) against the warp mma.sp kernel and the
oracle (marked gpu).

Both kernels multiply the same FP16 coefficients and FP16 high + residual panels with FP32
accumulation; only the order of the FP32 additions differs (one K = 32 tensor-core MMA per
tile here, the hi and residual products kept in separate accumulator columns and added at the
end).  Gates (written here): the two kernels' operator outputs within 1e-6 rel, the FP16x2
emulation within 2e-5 (the mma.sp kernel's gate), 10-iteration CG images within 2e-4 rel of
each other (CG amplifies the different FP32 summation orders) and within the 0.2% magnitude
NRMSE of the FP64 CG, residual histories of both kernels against the FP64 CG's (2e-3, and 2e-2
for the last two, tiny residuals of the undersampled case); repeated launches and graph
replays bitwise identical; the kernel's error word (a bounded wait that gave up) stays 0.
"""
import numpy as np
import pytest

from gpu_cases import case, measurement, oracle_cg, rel_l2, torch_inputs, volume_case
from oracle import nudft as onudft
from oracle import operator as oop
from trajsparsenufft_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CASES = ["grad4", "headline"]  # 8-coil image cases: 4x-undersampled and full radial


def _plans(name):
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, _ = case(name)
    kw = dict(im_size=n, grid_size=g, coils=c, width=j)
    return Plan.from_trajectory(traj, interp="tcgen05", **kw), Plan.from_trajectory(traj, interp="mma_sp", **kw)


@pytest.mark.parametrize("name", CASES)
def test_tc_forward_adjoint_match_mma_sp_and_emulation(name):
    traj, x, s, n, g, c, j, _ = case(name)
    tc, ref = _plans(name)
    assert tc.interp == "tcgen05" and ref.interp == "mma_sp"
    xt, st, _ = torch_inputs(name)
    y_tc, y_ref = tc.forward(xt, st), ref.forward(xt, st)
    rng = np.random.default_rng(5)
    yr = torch.from_numpy((rng.standard_normal((c, len(traj))) + 1j * rng.standard_normal((c, len(traj))))
                          .astype(np.complex64)).cuda()
    a_tc, a_ref = tc.adjoint(yr, st), ref.adjoint(yr, st)
    torch.cuda.synchronize()
    assert tc.device_error() == 0
    assert rel_l2(y_tc.cpu().numpy(), y_ref.cpu().numpy()) <= 1e-6
    assert rel_l2(a_tc.cpu().numpy(), a_ref.cpu().numpy()) <= 1e-6
    emu = oop.KbSenseOperator(traj, n, g, j, matrix_mode="fp16", panel_mode="split2", workers=8)
    assert rel_l2(y_tc.cpu().numpy(), emu.forward(x, s)) <= 2e-5
    assert rel_l2(a_tc.cpu().numpy(), emu.adjoint(yr.cpu().numpy(), s)) <= 2e-5
    # coil images in and out (no maps): the same views
    yc = tc.forward(torch.from_numpy((x[None] * s).astype(np.complex64)).cuda())
    assert rel_l2(yc.cpu().numpy(), y_tc.cpu().numpy()) <= 1e-5
    # repeated launches are bitwise identical (deterministic split-group reduction)
    np.testing.assert_array_equal(tc.forward(xt, st).cpu().numpy(), y_tc.cpu().numpy())
    np.testing.assert_array_equal(tc.adjoint(yr, st).cpu().numpy(), a_tc.cpu().numpy())


@pytest.mark.parametrize("name,density", [("grad4", False), ("headline", True)])
def test_tc_cg_sense_matches_mma_sp_and_fp64(name, density):
    traj, x, s, n, g, c, j, readout = case(name)
    tc, ref = _plans(name)
    _, st, yt = torch_inputs(name)
    w = synth.ramp_density(traj, readout) if density else None
    wt = None if w is None else torch.from_numpy(w).cuda()
    x_tc, h_tc, s_tc = tc.cg_sense(yt, st, density=wt, lam=1e-4, iters=10)
    assert s_tc["positive_curvature"] and s_tc["finite"] and not s_tc["timeout"]
    assert s_tc["completed_iterations"] == 10
    for _ in range(3):  # graph replays are bitwise identical (no race in the kernel's rings)
        x2, h2, _ = tc.cg_sense(yt, st, density=wt, lam=1e-4, iters=10)
        np.testing.assert_array_equal(x2.cpu().numpy(), x_tc.cpu().numpy())
        np.testing.assert_array_equal(h2, h_tc)
    assert tc.device_error() == 0
    x_ref, h_ref, _ = ref.cg_sense(yt, st, density=wt, lam=1e-4, iters=10)
    # ten CG iterations amplify the two kernels' different FP32 summation orders (3e-5 on the
    # image of the 4x-undersampled case); its last residual, 1e-3 of the first, moved by up to
    # 1.2%: the residual histories are compared with the FP64 CG's
    assert rel_l2(x_tc.cpu().numpy(), x_ref.cpu().numpy()) <= 2e-4
    op = oop.KbSenseOperator(traj, n, g, j, workers=8)
    x64, h64, _ = oracle_cg(lambda v: op.forward(v, s), lambda v: op.adjoint(v, s), measurement(name), w, 10, 1e-4)
    assert oop.magnitude_nrmse(x_tc.cpu().numpy(), x64) <= 2e-3
    e_tc = np.abs(np.asarray(h_tc) / np.asarray(h64) - 1)
    e_ref = np.abs(np.asarray(h_ref) / np.asarray(h64) - 1)
    assert e_tc[:-2].max() <= 2e-3 and e_ref[:-2].max() <= 2e-3
    assert e_tc.max() <= 2e-2 and e_ref.max() <= 2e-2, (e_tc, e_ref)


def test_tc_volume_matches_mma_sp():
    """A 64^3 kooshball with 8 coils: 3D views (2^21-cell grid rows) through the same kernel."""
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j = volume_case("vol64c8")
    kw = dict(im_size=n, grid_size=g, coils=c, width=j)
    tc, ref = Plan.from_trajectory(traj, interp="tcgen05", **kw), Plan.from_trajectory(traj, interp="mma_sp", **kw)
    xt, st = torch.from_numpy(x).cuda(), torch.from_numpy(s).cuda()
    y_tc, y_ref = tc.forward(xt, st), ref.forward(xt, st)
    a_tc, a_ref = tc.adjoint(y_ref, st), ref.adjoint(y_ref, st)
    torch.cuda.synchronize()
    assert tc.device_error() == 0
    # long items (cells near the centre of a kooshball are touched by many spokes) are summed
    # inside the tensor-core accumulator here and in registers there: FP32 order only
    assert rel_l2(y_tc.cpu().numpy(), y_ref.cpu().numpy()) <= 5e-6
    assert rel_l2(a_tc.cpu().numpy(), a_ref.cpu().numpy()) <= 5e-6
    emu = oop.KbSenseOperator3(traj, n, g, j, matrix_mode="fp16", panel_mode="split2", workers=8)
    assert rel_l2(y_tc.cpu().numpy(), emu.forward(x, s)) <= 2e-5


def test_tc_refused_where_not_built():
    """Four coils (16-half panel rows) and the complex reference-layout pack are not built for
    the tensor-core kernel: asking for it is refused; "auto" still plans."""
    from trajsparsenufft_b200._lib import TsnError
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, _ = case("small")
    with pytest.raises(TsnError) as info:
        Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j, interp="tcgen05")
    assert info.value.kind == "UNSUPPORTED"
    t8 = case("grad4")[0]
    with pytest.raises(TsnError):
        Plan.from_trajectory(t8, im_size=256, grid_size=512, coils=8, width=6, interp="tcgen05",
                             reference_layout=True)
    assert Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j, interp="auto").interp == "mma_sp"
