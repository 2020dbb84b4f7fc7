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


def test_noalloc_rejects_oversize_input(plfbs_lib):
    import torch

    res = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    rc = plfbs_lib.plfbs_residual_norms_noalloc(res.data_ptr(), MAX_CELLS + 1, 1.0, 0.1,
                                                out.data_ptr(), None)
    assert rc == capi.ERR_ARG
    assert b"8388608" in plfbs_lib.plfbs_last_error(None)
