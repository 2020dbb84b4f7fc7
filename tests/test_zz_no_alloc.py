"""plfbs_residual_norms_noalloc: the residual norms for callers that cannot let
the library allocate device memory (a fixed device-memory budget reserved at
start-up, or a host framework whose allocator must own every device byte).

Collected last on purpose. Device buffers here come from the caller side
(torch tensors); the entry point itself allocates nothing. Its output is
checked against the norms plfbs_run computes on the device for the same
residuals, on two calls in a row, within the tolerance of the stage tests.
"""

import numpy as np
import pytest

from conftest import rel_err
from plfbs import capi, cases

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the per-stage tolerance of test_gpu_parity.py
MAX_CELLS = 8388608


def _cavity(n=32):
    pm = cases.uniform_box(n, n, n, patch_types=["wall", "wall", "wall", "lid", "wall", "wall"])
    c = cases.Case(mesh_dir="", X=n, Y=n, Z=n, dt=0.18, mach=0.1, reynolds=100, ref_length=n,
                   bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann"),
                        cases.BC("lid", 1, 1, 0, 0, "dirichlet", "neumann")])
    return cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min), c


def test_noalloc_norms_match_run_twice(plfbs_lib):
    import torch

    ma, c = _cavity()  # 32,768 cells: 8 blocks of the static-scratch reduction
    rt, vt, val = cases.bc_arrays(ma, c)
    cfg = dict(visc=c.visc, dt=c.dt, max_velocity=c.mach, ref_rho=1.0, lengths=(c.X, c.Y, c.Z))
    s = capi.Solver(ma, rt, vt, val, cfg)
    s.set_debug(True)
    s0 = np.zeros((ma.total_cells, 4))
    s0[:, 3] = 1.0
    s.set_state(s0)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        stats, _ = s.run(1)  # the existing entry point: norms of the last RK stage
        res = torch.from_numpy(np.ascontiguousarray(s.residual())).cuda()
        out = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
        rc = plfbs_lib.plfbs_residual_norms_noalloc(res.data_ptr(), ma.n_cells, 1.0, c.mach,
                                                    out.data_ptr(), stream)
        assert rc == 0, plfbs_lib.plfbs_last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = np.array([stats["max_error"], stats["rho_rms"], stats["u_rms"], stats["v_rms"],
                         stats["w_rms"]])
        assert rel_err(got, want) < TOL, (call, got, want)
    s.close()


def _norms_numpy(res, ref_rho, u_ref):
    """The residual norms of residuals.cpp:95-147 in float64 numpy."""
    n = res.shape[0]
    rms = np.sqrt((res.astype(np.float64) ** 2).sum(axis=0) / n)  # u, v, w, rho
    rho = rms[3] / ref_rho
    u, v, w = rms[:3] / (ref_rho * u_ref)
    return np.array([max(w, u, v), rho, u, v, w])


@pytest.mark.parametrize("n", [4097, 1000003, MAX_CELLS])
def test_noalloc_random_sizes_no_device_memory(plfbs_lib, n):
    """Ragged and maximal sizes against numpy, twice in a row, with the device's
    free memory and torch's allocated bytes unchanged across the second call;
    the same residuals 8 bytes off a 32-byte boundary take the scalar loads."""
    import torch

    rng = np.random.Generator(np.random.PCG64(n))
    res_h = rng.standard_normal((n, 4)) * np.array([1e-3, 2e-3, 5e-4, 1e-4])
    want = _norms_numpy(res_h, 1.2, 0.05)
    buf = torch.zeros(4 * n + 4, dtype=torch.float64, device="cuda")
    buf[:4 * n] = torch.from_numpy(res_h.ravel()).cuda()
    out = torch.full((2, 5), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert buf.data_ptr() % 32 == 0
    for call in range(2):
        torch.cuda.synchronize()
        free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
        rc = plfbs_lib.plfbs_residual_norms_noalloc(buf.data_ptr(), n, 1.2, 0.05,
                                                    out[call].data_ptr(), stream)
        assert rc == 0, plfbs_lib.plfbs_last_error(None)
        torch.cuda.synchronize()
        if call == 1:  # the first call may load the library's device code
            assert torch.cuda.mem_get_info()[0] == free0
            assert torch.cuda.memory_allocated() == alloc0
        assert rel_err(out[call].cpu().numpy(), want) < TOL, (call, out[call], want)
    # unaligned: the same values one double further on
    buf[1:4 * n + 1] = torch.from_numpy(res_h.ravel()).cuda()
    rc = plfbs_lib.plfbs_residual_norms_noalloc(buf.data_ptr() + 8, n, 1.2, 0.05,
                                                out[0].data_ptr(), stream)
    assert rc == 0, plfbs_lib.plfbs_last_error(None)
    torch.cuda.synchronize()
    assert rel_err(out[0].cpu().numpy(), want) < TOL


def test_noalloc_rejects_oversize_input(plfbs_lib):
    import torch

    res = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    rc = plfbs_lib.plfbs_residual_norms_noalloc(res.data_ptr(), MAX_CELLS + 1, 1.0, 0.1,
                                                out.data_ptr(), None)
    assert rc == capi.ERR_ARG
    assert b"8388608" in plfbs_lib.plfbs_last_error(None)
