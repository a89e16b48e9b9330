"""GPU parity of the sm_100a operator pipeline against the oracle (marked gpu).

Tolerances (written here, from the reference gates where one exists):
* raw sparse interpolation vs reference.bin: max_abs <= 2e-2 and rel_l2 <= 2e-3
  (nufft_spmma_bench.cu:1102), and rel_l2 <= 1e-6 vs the exact FP64 product of the
  same FP16 coefficients and inputs;
* operator vs FP16x2 arithmetic emulation: rel_l2 <= 2e-5 (validate_fp16x2_native.py:247-253);
* operator vs FP64 direct NUDFT: rel_l2 <= 5e-4;
* adjointness |<y,Ax> - <A^H y,x>| / (|y| |Ax|) <= 1e-5;
* reconstruction magnitude NRMSE vs FP64 CG-SENSE <= 2e-3 (0.2%).
"""
import numpy as np
import pytest

from golden_io import GOLDEN
from gpu_cases import case, measurement, oracle_cg, rel_l2, torch_inputs
from oracle import nudft as onudft
from oracle import operator as oop
from oracle import planner as P

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _plan(name, **kw):
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, _ = case(name)
    return Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j, **kw)


@pytest.mark.parametrize("name", ["prod_radial16_opt", "prod_spiral32_opt"])
@pytest.mark.parametrize("view", ["G", "G_T"])
def test_raw_interpolation_matches_reference_bin(name, view):
    from trajsparsenufft_b200.operator import Plan
    import json
    root = GOLDEN / name
    spec = json.loads((root / "G" / "real" / "manifest.json").read_text())
    n, g = spec["im_size"], spec["grid_size"]
    plan = Plan.from_pack(root / "G" / "real", root / "G" / "imag", root / "G_T" / "real", root / "G_T" / "imag",
                          im_size=n, grid_size=g, coils=4, width=spec["numpoints"])
    for ci, comp in enumerate(("real", "imag")):
        d = root / view / comp
        dense = np.fromfile(d / "dense_input.bin", dtype=np.float16).reshape(-1, 16)
        ref = np.fromfile(d / "reference.bin", dtype=np.float32).reshape(-1, 16)
        out = plan.interp_component(view, ci, torch.from_numpy(dense).cuda()).cpu().numpy()
        err = np.abs(out - ref)
        assert err.max() <= 2e-2 and rel_l2(out, ref) <= 2e-3
        # exact product of the packed FP16 coefficients (csr_vals.bin) and the FP16 input
        rp = np.fromfile(d / "csr_row_ptr.bin", dtype=np.uint32).astype(np.int64)
        rid = np.fromfile(d / "csr_row_ids.bin", dtype=np.int32)
        cols = np.fromfile(d / "csr_cols.bin", dtype=np.int32)
        vals = np.fromfile(d / "csr_vals.bin", dtype=np.float16).astype(np.float64)
        exact = np.zeros_like(ref, dtype=np.float64)
        for r in range(len(rid)):
            sl = slice(rp[r], rp[r + 1])
            exact[rid[r]] = vals[sl] @ dense[cols[sl]].astype(np.float64)
        assert rel_l2(out, exact) <= 1e-6


@pytest.mark.parametrize("name,layout", [("small", "centered"), ("small", "reference"), ("n192", "centered"),
                                         ("n320", "reference")])
def test_forward_adjoint_match_oracle(name, layout):
    traj, x, s, n, g, c, j, _ = case(name)
    plan = _plan(name, reference_layout=(layout == "reference"))
    xt, st, _ = torch_inputs(name)
    y_gpu = plan.forward(xt, st).cpu().numpy()
    emu = oop.KbSenseOperator(traj, n, g, j, matrix_mode="fp16", panel_mode="split2")
    ex = onudft.Nudft(traj, n)
    assert rel_l2(y_gpu, emu.forward(x, s)) <= 2e-5
    assert rel_l2(y_gpu, ex.forward(x, s)) <= 5e-4
    rng = np.random.default_rng(11)
    yr = (rng.standard_normal((c, len(traj))) + 1j * rng.standard_normal((c, len(traj)))).astype(np.complex64)
    a_gpu = plan.adjoint(torch.from_numpy(yr).cuda(), st).cpu().numpy()
    assert rel_l2(a_gpu, emu.adjoint(yr, s)) <= 2e-5
    assert rel_l2(a_gpu, ex.adjoint(yr, s)) <= 5e-4
    # coil-image variants (smaps = NULL)
    coil = (x[None] * s).astype(np.complex64)
    yc = plan.forward(torch.from_numpy(coil).cuda()).cpu().numpy()
    assert rel_l2(yc, y_gpu) <= 1e-5
    ac = plan.adjoint(torch.from_numpy(yr).cuda()).cpu().numpy()
    assert rel_l2(ac, ex.adjoint(yr)) <= 5e-4
    # adjointness of the FP16x2 pair
    left = np.vdot(y_gpu.astype(np.complex128), yr)
    right = np.vdot(x.astype(np.complex128), a_gpu)
    gap = abs(left - right) / (np.linalg.norm(yr) * np.linalg.norm(y_gpu))
    assert gap <= 1e-5


def test_headline_operator_accuracy():
    """The headline shape (256^2 image, 512^2 grid, 8 coils, 131072 samples, J = 6) through the
    product's default plan: forward and adjoint against the FP16x2 emulation (<= 2e-5), the FP64
    KB operator (<= 5e-4) and the FP64 direct NUDFT (forward on every 64th sample, adjoint in
    full; <= 5e-4), and the adjointness gap of the FP16x2 pair (<= 1e-5)."""
    traj, x, s, n, g, c, j, _ = case("headline")
    plan = _plan("headline")
    xt, st, _ = torch_inputs("headline")
    emu = oop.KbSenseOperator(traj, n, g, j, matrix_mode="fp16", panel_mode="split2", workers=8)
    f64 = oop.KbSenseOperator(traj, n, g, j, workers=8)
    y_gpu = plan.forward(xt, st).cpu().numpy()
    assert rel_l2(y_gpu, emu.forward(x, s)) <= 2e-5
    assert rel_l2(y_gpu, f64.forward(x, s)) <= 5e-4
    sub = np.arange(0, len(traj), 64)
    assert rel_l2(y_gpu[:, sub], onudft.Nudft(traj[sub], n).forward(x, s)) <= 5e-4
    rng = np.random.default_rng(12)
    yr = (rng.standard_normal((c, len(traj))) + 1j * rng.standard_normal((c, len(traj)))).astype(np.complex64)
    a_gpu = plan.adjoint(torch.from_numpy(yr).cuda(), st).cpu().numpy()
    assert rel_l2(a_gpu, emu.adjoint(yr, s)) <= 2e-5
    assert rel_l2(a_gpu, f64.adjoint(yr, s)) <= 5e-4
    assert rel_l2(a_gpu, onudft.Nudft(traj, n).adjoint(yr, s)) <= 5e-4
    left = np.vdot(y_gpu.astype(np.complex128), yr)
    right = np.vdot(x.astype(np.complex128), a_gpu)
    assert abs(left - right) / (np.linalg.norm(yr) * np.linalg.norm(y_gpu)) <= 1e-5


def test_pack_dirs_drop_in_matches_trajectory_plan(tmp_path):
    """Reference-format directories (written by our planner) load as a drop-in and give
    bit-identical results to the in-memory reference-layout plan."""
    from trajsparsenufft_b200 import packing
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, _ = case("small")
    dirs = packing.export_production(traj, tmp_path, im_size=n, grid_size=g, width=j)
    p1 = Plan.from_pack(dirs["G"] / "real", dirs["G"] / "imag", dirs["G_T"] / "real", dirs["G_T"] / "imag",
                        im_size=n, grid_size=g, coils=c, width=j)
    p2 = _plan("small", reference_layout=True)
    xt, st, yt = torch_inputs("small")
    np.testing.assert_array_equal(p1.forward(xt, st).cpu().numpy(), p2.forward(xt, st).cpu().numpy())
    np.testing.assert_array_equal(p1.adjoint(yt, st).cpu().numpy(), p2.adjoint(yt, st).cpu().numpy())


@pytest.mark.parametrize("name", ["cfg0"])
def test_cg_sense_cfg0_matches_fp64_nudft(name):
    traj, x, s, n, g, c, j, readout = case(name)
    plan = _plan(name)
    xt, st, yt = torch_inputs(name)
    from trajsparsenufft_b200 import synth
    w = synth.ramp_density(traj, readout)
    wt = torch.from_numpy(w).cuda()
    lam = 1e-4
    x_gpu, hist, status = plan.cg_sense(yt, st, density=wt, lam=lam, iters=10)
    x_gpu = x_gpu.cpu().numpy()
    assert status["positive_curvature"] and status["finite"] and status["completed_iterations"] == 10
    nd = onudft.Nudft(traj, n)
    y = measurement(name)
    x_ref, res_ref, st_ref = oracle_cg(lambda v: nd.forward(v, s), lambda v: nd.adjoint(v, s), y, w, 10, lam)
    assert oop.magnitude_nrmse(x_gpu, x_ref) <= 2e-3
    assert rel_l2(x_gpu, x_ref) <= 2e-3
    # residual history follows the FP64 recursion
    np.testing.assert_allclose(hist, res_ref, rtol=2e-3)
    # graph replay is bitwise deterministic
    x2, _, _ = plan.cg_sense(yt, st, density=wt, lam=lam, iters=10)
    np.testing.assert_array_equal(x2.cpu().numpy(), x_gpu)


def test_cg_sense_headline_matches_fp64_kb():
    """Headline CG-SENSE (k-space from the direct FP64 NUDFT plus noise) against the FP64 KB
    CG on the same data: magnitude NRMSE within the 0.2% gate."""
    traj, x, s, n, g, c, j, _ = case("headline")
    plan = _plan("headline")
    xt, st, yt = torch_inputs("headline")
    x_gpu, hist, status = plan.cg_sense(yt, st, lam=1e-4, iters=10)
    assert status["positive_curvature"] and status["finite"]
    op = oop.KbSenseOperator(traj, n, g, j, workers=8)
    y = measurement("headline")
    x_ref, res_ref, _ = oracle_cg(lambda v: op.forward(v, s), lambda v: op.adjoint(v, s), y, None, 10, 1e-4)
    assert oop.magnitude_nrmse(x_gpu.cpu().numpy(), x_ref) <= 2e-3


@pytest.mark.parametrize("layout", ["reference", "centered"])
def test_cg_sense_matches_the_reference_solver_output(layout):
    """The GPU CG-SENSE against what the reference's own reference_sparse_solver computed
    (tests/golden/solver_small.npz, fp16x2 variant: FP16 matrix, FP16 high + residual panels,
    10 iterations; the fixture's power-of-two rescaling undone).  With the reference's complex
    pack layout the coefficients round to FP16 exactly as there: image within 2e-4 rel and
    residual history within 2e-3.  The centred real pack rounds different coefficients
    (the phase moved into the FFT): magnitude NRMSE within the 0.2% gate."""
    from golden_io import GOLDEN
    from trajsparsenufft_b200.operator import Plan
    d = np.load(GOLDEN / "solver_small.npz")
    n, g, c, j, iters = (int(v) for v in d["shape"])
    a, k = int(d["fp16x2_maps_scale_exp"]), int(d["fp16x2_data_scale_exp"])
    want = d["x_fp16x2"] * 2.0 ** (a - k)
    plan = Plan.from_trajectory(d["trajectory"], im_size=n, grid_size=g, coils=c, width=j,
                                reference_layout=(layout == "reference"))
    x_gpu, hist, status = plan.cg_sense(torch.from_numpy(d["data"]).cuda(), torch.from_numpy(d["smaps"]).cuda(),
                                        lam=float(d["lam"]), iters=iters)
    assert status["positive_curvature"] and status["finite"] and status["completed_iterations"] == iters
    x_gpu = x_gpu.cpu().numpy()
    assert oop.magnitude_nrmse(x_gpu, want) <= 2e-3
    if layout == "reference":
        assert rel_l2(x_gpu, want) <= 2e-4
        np.testing.assert_allclose(hist, d["residuals_fp16x2"] * 2.0 ** -(a + k), rtol=2e-3)


def test_cg_curvature_failure_is_reported_not_trapped():
    """A negative Tikhonov weight makes the normal operator indefinite: the status word
    reports the non-positive curvature and the iteration count stops before the failing
    iteration (0 here: the first denominator is already negative), as the reference solver
    stops there (reference_sparse_solver.py:281-287); nothing traps."""
    plan = _plan("small")
    _, st, yt = torch_inputs("small")
    for iters in (1, 3):
        x, hist, status = plan.cg_sense(yt, st, lam=-1e12, iters=iters)
        assert status["positive_curvature"] is False
        assert status.get("failure") == "CURVATURE"
        assert status["completed_iterations"] == 0, status


def test_misaligned_device_arrays_are_rejected():
    """The FFT stages stream images and maps with 16-byte copies: an array that starts
    8 bytes into an allocation is refused with an argument error before any launch."""
    from trajsparsenufft_b200._lib import TsnError
    plan = _plan("small")
    xt, st, yt = torch_inputs("small")
    n = plan.im_size
    buf = torch.zeros(n * n + 1, dtype=torch.complex64, device="cuda")
    x_off = buf[1:].view(n, n)
    assert x_off.data_ptr() % 16 == 8
    with pytest.raises(TsnError, match="16-byte aligned") as info:
        plan.forward(x_off, st)
    assert info.value.kind == "ARG"
    y = plan.forward(xt, st)  # the plan stays usable
    assert torch.isfinite(torch.view_as_real(y)).all()


@pytest.mark.parametrize("iters", [20, 50])
def test_long_cg_stays_on_the_fp64_path(iters):
    """Long CG (the reference's long-CG stability check, tools/check_long_cg.py:11-27): at 20 and
    50 iterations the FP16x2 solve stays finite with positive curvature and its image matches
    the FP64 CG at the same iteration count within the 0.2% magnitude NRMSE gate."""
    name = "cfg0"
    traj, x, s, n, g, c, j, readout = case(name)
    plan = _plan(name)
    _, st, yt = torch_inputs(name)
    from trajsparsenufft_b200 import synth
    w = synth.ramp_density(traj, readout)
    x_gpu, hist, status = plan.cg_sense(yt, st, density=torch.from_numpy(w).cuda(), lam=1e-4, iters=iters)
    assert status["positive_curvature"] and status["finite"] and status["completed_iterations"] == iters
    assert np.all(np.isfinite(hist)) and hist[-1] < hist[0]
    nd = onudft.Nudft(traj, n)
    x_ref, _, _ = oracle_cg(lambda v: nd.forward(v, s), lambda v: nd.adjoint(v, s), measurement(name), w, iters, 1e-4)
    assert oop.magnitude_nrmse(x_gpu.cpu().numpy(), x_ref) <= 2e-3


def test_fused_update_residual_matches_the_direct_norm():
    """The fused CG update takes rho' from an expansion over the stored r and Ap; the last
    iteration of a solve sums |r|^2 directly instead.  A solve of k iterations therefore ends
    on the direct norm of r_k, and a solve of k + 1 iterations reaches r_k through the
    expansion: the two residuals agree to FP32 rounding late into the solve (rtol 1e-3 on
    |r|), because each expansion restarts from the direct <r, r> of the previous iteration."""
    name = "cfg0"
    traj, x, s, n, g, c, j, readout = case(name)
    plan = _plan(name)
    _, st, yt = torch_inputs(name)
    from trajsparsenufft_b200 import synth
    w = torch.from_numpy(synth.ramp_density(traj, readout)).cuda()
    for k in (10, 30):
        _, hist_k, _ = plan.cg_sense(yt, st, density=w, lam=1e-4, iters=k)
        _, hist_k1, _ = plan.cg_sense(yt, st, density=w, lam=1e-4, iters=k + 1)
        assert hist_k[-1] < 1e-2 * hist_k[0]
        np.testing.assert_allclose(hist_k1[:k + 1], hist_k[:k + 1], rtol=1e-3)


def _oracle_reliable_cg(fwd, adj, y, w, iters, lam, period, direction):
    """FP64 restatement of the reference's reliable-update CG (reference_sparse_solver.py:200-332)."""
    wy = y if w is None else y * w[None]
    M = lambda v: adj(fwd(v) * (1.0 if w is None else w[None])) + lam * v
    b = adj(wy)
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rs_old = np.vdot(r, r).real
    res = [np.sqrt(rs_old)]
    for it in range(iters):
        ap = M(p)
        alpha = rs_old / np.vdot(p, ap).real
        x = x + alpha * p
        r = r - alpha * ap
        rs_new = np.vdot(r, r).real
        if period > 0 and (it + 1) % period == 0 and it + 1 < iters:
            r = b - M(x)
            rs_new = np.vdot(r, r).real
            p = r.copy() if direction == "restart" else r + (rs_new / rs_old) * p
        else:
            p = r + (rs_new / rs_old) * p
        res.append(np.sqrt(rs_new))
        rs_old = rs_new
    return x, np.array(res)


@pytest.mark.parametrize("direction", ["restart", "beta"])
def test_reliable_update_cg_matches_fp64(direction):
    name = "cfg0"
    traj, x, s, n, g, c, j, readout = case(name)
    plan = _plan(name)
    _, st, yt = torch_inputs(name)
    from trajsparsenufft_b200 import synth
    w = synth.ramp_density(traj, readout)
    iters, period = 30, 10
    x_gpu, hist, status = plan.cg_sense(yt, st, density=torch.from_numpy(w).cuda(), lam=1e-4, iters=iters,
                                        reliable_update_period=period, reliable_update_direction=direction)
    assert status["positive_curvature"] and status["finite"] and status["completed_iterations"] == iters
    nd = onudft.Nudft(traj, n)
    x_ref, res_ref = _oracle_reliable_cg(lambda v: nd.forward(v, s), lambda v: nd.adjoint(v, s), measurement(name),
                                         w.astype(np.float64), iters, 1e-4, period, direction)
    assert oop.magnitude_nrmse(x_gpu.cpu().numpy(), x_ref) <= 2e-3
    # the replaced residuals (after iterations 10 and 20) follow the FP64 reliable residuals
    np.testing.assert_allclose(hist[[period, 2 * period]], res_ref[[period, 2 * period]], rtol=2e-2)
    np.testing.assert_allclose(hist[:period], res_ref[:period], rtol=2e-3)


def test_reference_operator_is_fp32_class():
    """tsn_forward_reference / tsn_adjoint_reference (the reference's forward_reference /
    adjoint_reference): every KB weight as FP16 high part + FP16 residual, FP16x2 panels, FP32
    FFTs.  Gates: within 1e-6 rel of the FP64 KB operator (its emulation is 5e-8 away; the
    FP16-weight operator is 7e-5 away) and of the oracle's emulation of the same split; the plain
    operators of the same plan stay the FP16-weight ones; plans without the views refuse."""
    from trajsparsenufft_b200._lib import TsnError
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, readout = case("cfg0")
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j, reference_steps=True)
    xt, st, _ = torch_inputs("cfg0")
    rng = np.random.default_rng(11)
    yr = (rng.standard_normal((c, len(traj))) + 1j * rng.standard_normal((c, len(traj)))).astype(np.complex64)
    yt = torch.from_numpy(yr).cuda()
    f64 = oop.KbSenseOperator(traj, n, g, j, workers=8)
    ref = oop.KbSenseOperator(traj, n, g, j, matrix_mode="fp16x2", panel_mode="split2", workers=8)
    emu = oop.KbSenseOperator(traj, n, g, j, matrix_mode="fp16", panel_mode="split2", workers=8)
    y_ref, a_ref = plan.forward(xt, st, reference=True), plan.adjoint(yt, st, reference=True)
    y_pl, a_pl = plan.forward(xt, st), plan.adjoint(yt, st)
    torch.cuda.synchronize()
    y64, a64 = f64.forward(x, s), f64.adjoint(yr, s)
    errs = {"fwd_ref_vs_f64": rel_l2(y_ref.cpu().numpy(), y64), "adj_ref_vs_f64": rel_l2(a_ref.cpu().numpy(), a64),
            "fwd_ref_vs_emu": rel_l2(y_ref.cpu().numpy(), ref.forward(x, s)),
            "adj_ref_vs_emu": rel_l2(a_ref.cpu().numpy(), ref.adjoint(yr, s)),
            "fwd_plain_vs_f64": rel_l2(y_pl.cpu().numpy(), y64), "adj_plain_vs_f64": rel_l2(a_pl.cpu().numpy(), a64)}
    print(errs)
    assert max(errs["fwd_ref_vs_f64"], errs["adj_ref_vs_f64"], errs["fwd_ref_vs_emu"], errs["adj_ref_vs_emu"]) <= 1e-6, errs
    assert rel_l2(y_pl.cpu().numpy(), emu.forward(x, s)) <= 2e-5
    assert rel_l2(a_pl.cpu().numpy(), emu.adjoint(yr, s)) <= 2e-5
    with pytest.raises(TsnError, match="TSN_FLAG_REFERENCE_STEPS"):
        _plan("cfg0").forward(xt, st, reference=True)


def test_reference_steps_follow_the_reference_schedule():
    """Scheduled reference steps (reference_sparse_solver.py cg_sense: scheduled_reference_period,
    explicit_reference_steps): on a plan built with reference_steps=True, the chosen iterations
    apply the normal operator through the FP32-class views, and so does the right-hand side.
    Gates: a mixed schedule (every 3rd iteration and iteration 5) and an all-reference schedule
    match the oracle's restatement of the schedule (FP64 CG over the emulated operators) within
    1e-4 rel, with residual histories within 2e-3 (2e-2 for the last two, small residuals of the
    undersampled case) -- the FP32 vectors of the device CG, not the operators, set that floor;
    asking for reference steps on a plan without them is an argument error."""
    from trajsparsenufft_b200._lib import TsnError
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, readout = case("cfg0")
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j, reference_steps=True)
    _, st, yt = torch_inputs("cfg0")
    y = measurement("cfg0")
    f64 = oop.KbSenseOperator(traj, n, g, j, workers=8)
    emu = oop.KbSenseOperator(traj, n, g, j, matrix_mode="fp16", panel_mode="split2", workers=8)
    ref = oop.KbSenseOperator(traj, n, g, j, matrix_mode="fp16x2", panel_mode="split2", workers=8)
    x64, _, _ = oop.cg_sense(lambda v: f64.forward(v, s), lambda v: f64.adjoint(v, s), y, 10, 1e-4)
    report = {}
    for period, steps in ((1, ()), (3, (5,)), (0, (2, 7))):
        xg, hg, sg = plan.cg_sense(yt, st, lam=1e-4, iters=10, scheduled_reference_period=period,
                                   reference_steps=steps)
        assert sg["positive_curvature"] and sg["finite"] and sg["completed_iterations"] == 10
        xo, ho, so = oop.cg_sense_scheduled(
            lambda v: emu.forward(v, s), lambda v: emu.adjoint(v, s), lambda v: ref.forward(v, s),
            lambda v: ref.adjoint(v, s), y, 10, 1e-4, scheduled_reference_period=period,
            explicit_reference_steps=steps)
        e = rel_l2(xg.cpu().numpy(), xo)
        eh = np.abs(np.asarray(hg) / np.asarray(ho) - 1)
        report[(period, steps)] = (so["scheduled_reference_steps"], e, rel_l2(xg.cpu().numpy(), x64), eh.max())
        assert e <= 1e-4, report
        assert eh[:-2].max() <= 2e-3 and eh.max() <= 2e-2, report
    print(report)
    assert report[(3, (5,))][0] == [3, 5, 6, 9] and report[(0, (2, 7))][0] == [2, 7]
    x_plain, _, _ = plan.cg_sense(yt, st, lam=1e-4, iters=10)
    x_again, _, _ = _plan("cfg0").cg_sense(yt, st, lam=1e-4, iters=10)
    # the plain solve of a plan with reference views is the plain solve
    np.testing.assert_array_equal(x_plain.cpu().numpy(), x_again.cpu().numpy())
    with pytest.raises(TsnError, match="TSN_FLAG_REFERENCE_STEPS"):
        _plan("cfg0").cg_sense(yt, st, lam=1e-4, iters=10, scheduled_reference_period=2)
