"""Batched CG-SENSE over uneven plans (tsn_batch_*), marked gpu.

Every case of a batch runs the same per-item arithmetic as its own tsn_cg_sense call (the
FFT items and the interpolation work items are fixed per plan; only how many CTAs or warps
share them changes), so each batched reconstruction must equal the single-case one bit for
bit, and match the FP64 CG-SENSE oracle within the 0.2% magnitude NRMSE gate.
"""
import numpy as np
import pytest

from gpu_cases import case, measurement, oracle_cg, torch_inputs
from oracle import nudft as onudft
from oracle import operator as oop
from trajsparsenufft_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CASES = ["small", "cfg0", "n192", "c16"]


def _plan(name):
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, _ = case(name)
    return Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j)


def test_batch_matches_single_case_solves_bitwise():
    from trajsparsenufft_b200.operator import Batch
    plans = [_plan(nm) for nm in CASES]
    ys, maps, dens = [], [], []
    for nm in CASES:
        _, st, yt = torch_inputs(nm)
        ys.append(yt)
        maps.append(st)
        traj = case(nm)[0]
        dens.append(torch.from_numpy(synth.ramp_density(traj, case(nm)[7])).cuda() if nm == "cfg0" else None)
    singles = []
    for pl, y, s, w in zip(plans, ys, maps, dens):
        x, _, status = pl.cg_sense(y, s, density=w, lam=1e-4, iters=10)
        assert status["positive_curvature"] and status["finite"]
        singles.append(x.clone())
    batch = Batch(plans, streams=3)
    for _ in range(2):  # the second call replays the captured graph
        xs, statuses = batch.cg_sense(ys, maps, densities=dens, lam=1e-4, iters=10)
        for nm, xb, xs1, st in zip(CASES, xs, singles, statuses):
            assert st["completed_iterations"] == 10 and st["positive_curvature"] and st["finite"], nm
            assert torch.equal(xb, xs1), nm


def test_batch_cases_match_fp64_oracle():
    from trajsparsenufft_b200.operator import Batch
    names = ["small", "n192"]
    plans = [_plan(nm) for nm in names]
    ins = [torch_inputs(nm) for nm in names]
    xs, statuses = Batch(plans).cg_sense([i[2] for i in ins], [i[1] for i in ins], lam=1e-4, iters=10)
    for nm, xb in zip(names, xs):
        traj, x, s, n, *_ = case(nm)
        ex = onudft.Nudft(traj, n)
        x_ref, _, _ = oracle_cg(lambda v: ex.forward(v, s), lambda v: ex.adjoint(v, s), measurement(nm), None, 10,
                                1e-4)
        assert oop.magnitude_nrmse(xb.cpu().numpy(), x_ref) <= 2e-3, nm


def test_batch_rejects_bad_arguments():
    from trajsparsenufft_b200._lib import TsnError
    from trajsparsenufft_b200.operator import Batch
    plan = _plan("small")
    _, st, yt = torch_inputs("small")
    b = Batch([plan])
    with pytest.raises(ValueError):
        b.cg_sense([yt, yt], [st], lam=1e-4, iters=2)
    n = plan.im_size
    buf = torch.zeros(n * n + 1, dtype=torch.complex64, device="cuda")
    with pytest.raises(TsnError, match="16-byte aligned"):
        b.cg_sense([yt], [st], outs=[buf[1:].view(n, n)], lam=1e-4, iters=2)
