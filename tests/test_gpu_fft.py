"""FFT endpoints vs numpy FFTs (marked gpu).

Gates from the reference's custom-FFT self checks (nufft_integrated_bench.cu:1217-1237,
:1264-1280): forward panel rel_l2 <= 5e-4, inverse rel_l2 <= 2e-5.  The FP16 high +
residual panel carries ~2^-22 relative precision, so the forward is held to 1e-5 here.
"""
import numpy as np
import pytest

from gpu_cases import case, rel_l2
from oracle import kb as okb

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _grid_from_image(img, g, shift):
    """[C, G, G] padded grid: position n holds image index (n + shift) mod G (if < N)."""
    c, n, _ = img.shape
    out = np.zeros((c, g, g), dtype=np.complex128)
    pos = (np.arange(n) - shift) % g
    out[:, pos[:, None], pos[None, :]] = img
    return out


@pytest.mark.parametrize("name,layout", [("small", "centered"), ("small", "reference"), ("cfg0", "centered"),
                                         ("headline", "centered"), ("c16", "reference"), ("n192", "centered"),
                                         ("n320", "reference")])
def test_forward_panel_matches_numpy_fft(name, layout):
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, _ = case(name)
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j,
                                reference_layout=(layout == "reference"))
    panel, scale = plan.fft_forward_panel(torch.from_numpy(x).cuda(), torch.from_numpy(s).cuda())
    p = panel.float().cpu().numpy().astype(np.float64)            # [G*G, 4C], rows q1*G + q0
    hi, res = p[:, : 2 * c], p[:, 2 * c:]
    v = (hi + res)[:, 0::2] + 1j * (hi + res)[:, 1::2]            # [G*G, C]
    got = v.reshape(g, g, c).transpose(2, 1, 0) / scale           # [C, q0, q1]
    d = okb.deapodization(n, g, j)
    shift = 0 if layout == "reference" else n // 2
    want = np.fft.fft2(_grid_from_image(x[None] * s * d[None], g, shift))
    assert rel_l2(got, want) <= 1e-5


@pytest.mark.parametrize("name,layout", [("small", "centered"), ("cfg0", "reference"), ("headline", "centered"),
                                         ("c16", "centered"), ("n192", "reference"), ("n320", "centered")])
def test_adjoint_endpoint_matches_numpy_ifft(name, layout):
    from trajsparsenufft_b200.operator import Plan
    traj, x, s, n, g, c, j, _ = case(name)
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=j,
                                reference_layout=(layout == "reference"))
    rng = np.random.default_rng(5)
    grid = (rng.standard_normal((c, g, g)) + 1j * rng.standard_normal((c, g, g))).astype(np.complex64)
    internal = np.ascontiguousarray(grid.transpose(2, 1, 0).reshape(g * g, c))   # rows q1*G + q0
    st = torch.from_numpy(s).cuda()
    got = plan.fft_adjoint_image(torch.from_numpy(internal).cuda(), st).cpu().numpy()
    coils = plan.fft_adjoint_image(torch.from_numpy(internal).cuda()).cpu().numpy()
    d = okb.deapodization(n, g, j)
    shift = 0 if layout == "reference" else n // 2
    full = np.fft.ifft2(grid.astype(np.complex128)) * g * g
    pos = (np.arange(n) - shift) % g
    img = full[:, pos[:, None], pos[None, :]] * d[None]
    assert rel_l2(coils, img) <= 2e-5
    assert rel_l2(got, np.sum(np.conj(s) * img, axis=0)) <= 2e-5
