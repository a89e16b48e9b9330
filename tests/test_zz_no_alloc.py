"""The allocation-free adjoint FFT endpoint (marked gpu; collected last on purpose).

tsn_fft_adjoint_image_static serves callers that cannot call cudaMalloc (frozen
allocators, fully pre-reserved device memory, plug-ins inside an application that owns
the device memory): it takes all inputs and outputs from the caller and keeps its
intermediate in a fixed device array.  These tests call it through the C ABI and check
the results against the plan-based endpoint tsn_fft_adjoint_image on the same inputs,
rel_l2 <= 1e-6 (both run the same FP32 kernels): twice in a row, and alternating grid
sizes in stream order on a non-blocking stream with free device memory unchanged.
They run standalone in a fresh process as well as after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("centered", [True, False])
def test_static_adjoint_endpoint_matches_plan_endpoint(centered):
    from trajsparsenufft_b200 import _lib, packing, synth
    from trajsparsenufft_b200.operator import Plan

    n, g, c = 128, 256, 8
    traj = synth.golden_radial(32, 256)
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=6, reference_layout=not centered)
    s = torch.from_numpy(synth.coil_maps(n, c, 7)).cuda()
    scaling = torch.from_numpy(packing.kb_deapodization(n, g, 6).astype(np.float32)).cuda()
    rng = np.random.default_rng(21)
    L = _lib.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        grid = (rng.standard_normal((g * g, c)) + 1j * rng.standard_normal((g * g, c))).astype(np.complex64)
        gt = torch.from_numpy(grid).cuda()
        want = plan.fft_adjoint_image(gt, s).cpu().numpy()
        out = torch.empty((n, n), dtype=torch.complex64, device="cuda")
        rc = L.tsn_fft_adjoint_image_static(n, g, c, int(centered), C.c_void_p(gt.data_ptr()),
                                            C.c_void_p(s.data_ptr()), C.c_void_p(scaling.data_ptr()),
                                            C.c_void_p(out.data_ptr()), stream)
        _lib.check(rc)
        torch.cuda.synchronize()
        assert _rel(out.cpu().numpy(), want) <= 1e-6, f"call {call}"


def test_static_adjoint_endpoint_rejects_oversized_shapes():
    from trajsparsenufft_b200 import _lib
    L = _lib.lib()
    dummy = torch.zeros(16, dtype=torch.complex64, device="cuda")
    p = C.c_void_p(dummy.data_ptr())
    rc = L.tsn_fft_adjoint_image_static(512, 1024, 16, 1, p, p, C.c_void_p(dummy.data_ptr()), p, None)
    assert _lib.STATUS[rc] == "SHAPE"
    assert b"exceeds the static scratch" in L.tsn_get_last_error_string()


def test_static_adjoint_endpoint_alternating_grids_on_one_stream():
    """Calls of grid sizes 256 and 512 queued back to back on one non-blocking stream (no
    host synchronization between them) each match the plan endpoint, and free device memory
    is the same before and after the queued calls."""
    from trajsparsenufft_b200 import _lib, packing, synth
    from trajsparsenufft_b200.operator import Plan

    c = 8
    L = _lib.lib()
    stream = torch.cuda.Stream()  # non-blocking with respect to the legacy default stream
    cases = []
    rng = np.random.default_rng(33)
    for n, g in ((128, 256), (256, 512)):
        traj = synth.golden_radial(32, 2 * n)
        plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=6)
        s = torch.from_numpy(synth.coil_maps(n, c, 9)).cuda()
        scaling = torch.from_numpy(packing.kb_deapodization(n, g, 6).astype(np.float32)).cuda()
        grid = torch.from_numpy((rng.standard_normal((g * g, c))
                                 + 1j * rng.standard_normal((g * g, c))).astype(np.complex64)).cuda()
        want = plan.fft_adjoint_image(grid, s).cpu().numpy()
        cases.append((n, g, s, scaling, grid, want))
    sched = [0, 1, 0, 1, 1, 0]
    outs = [torch.empty((cases[i][0],) * 2, dtype=torch.complex64, device="cuda") for i in sched]
    torch.cuda.synchronize()

    def queue():
        for i, out in zip(sched, outs):
            n, g, s, scaling, grid, _ = cases[i]
            _lib.check(L.tsn_fft_adjoint_image_static(n, g, c, 1, C.c_void_p(grid.data_ptr()),
                                                      C.c_void_p(s.data_ptr()), C.c_void_p(scaling.data_ptr()),
                                                      C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream)))

    queue()  # first calls: set-up and lazy kernel loading happen here
    stream.synchronize()
    for out in outs:
        out.zero_()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    queue()
    stream.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    for k, (i, out) in enumerate(zip(sched, outs)):
        assert _rel(out.cpu().numpy(), cases[i][5]) <= 1e-6, f"call {k} (grid {cases[i][1]})"
