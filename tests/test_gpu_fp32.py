"""The FP32 deviation form (PLFBS_FP32_DEVIATION) against the FP64 reference.

State, gradients, fluxes, geometry and weights in FP32 with rho stored as
rho - rho0 and velocity divided by U; residual norms in FP64. There is no
bit-level bar: the tests bound the error against the FP64 golden fixtures
(the reference's own kernels) and the FP64 oracle, per field, at levels FP32
rounding of O(1e-7) relative explains with margin.
"""

import numpy as np
import pytest

import golden_cases
import oracle
from conftest import load_golden, rel_err, rel_l2
from plfbs import capi, cases

pytestmark = pytest.mark.gpu

STAGE_TOL = 1e-4   # one stage, max relative error of each quantity
RUN_TOL = 2e-5     # whole runs, relative L2 of each field


def _solver32(d, **over):
    cfg = golden_cases.oracle_cfg(d)
    cfg.update(over)
    cfg["precision"] = capi.FP32_DEVIATION
    cfg["renumber"] = 1
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    ibm = dict(node_ref=d["nodes"], stiffness=cfg["stiffness"], radius=cfg["radius"],
               depth=cfg["depth"], object_nodes=cfg["object_nodes"])
    return capi.Solver(d["ma"], rt, vt, val, cfg, ibm=ibm)


def _field_errors(st, ref):
    # velocity relative to its own scale; density through rho - rho0
    out = {}
    for k, name in enumerate(("u", "v", "w")):
        out[name] = rel_l2(st[:, k], ref[:, k])
    out["rho-rho0"] = rel_l2(st[:, 3] - 1.0, ref[:, 3] - 1.0)
    return out


@pytest.mark.parametrize("name", golden_cases.NAMES)
def test_fp32_first_stage(plfbs_lib, name):
    d = golden_cases.build(name)
    g = load_golden(name)
    C = d["ma"].n_cells
    s = _solver32(d)
    s.set_debug(True)
    s.set_state(d["state0"])
    s.run_stages(1)
    st = s.get_state()
    assert rel_err(s.gradients(), g["s0_grad"][:C]) < STAGE_TOL
    assert rel_err(s.face_flux(), g["s0_face_flux"]) < STAGE_TOL
    assert rel_err(s.residual(), g["s0_residual"]) < STAGE_TOL
    assert rel_err(st[:C, :3], g["s0_state_rk"][:C, :3]) < STAGE_TOL
    assert rel_err(st[:C, 3] - 1.0, g["s0_state_rk"][:C, 3] - 1.0) < STAGE_TOL
    x, v, f = s.nodes()
    assert rel_err(x, g["s0_nodes"][:, 0:3]) < 1e-9  # positions stay FP64
    s.close()


@pytest.mark.parametrize("name", ["cavity", "channel", "graded"])
def test_fp32_run(plfbs_lib, name):
    d = golden_cases.build(name)
    g = load_golden(name)
    s = _solver32(d)
    s.set_state(d["state0"])
    stats, hist = s.run(d["case"].steps)
    errs = _field_errors(s.get_state(), g["final_state"])
    assert max(errs.values()) < RUN_TOL, errs
    assert rel_err(hist[:, 1:], g["history"][:, 1:]) < 1e-3


def test_fp32_cavity_32cubed(plfbs_lib):
    """The 32^3 lid-driven cavity from rest, 50 steps, FP32 deviation form
    against the FP64 oracle: per-field relative L2 error."""
    n = 32
    pm = cases.uniform_box(n, n, n, patch_types=["wall", "wall", "wall", "lid", "wall", "wall"])
    c = cases.Case(mesh_dir="", X=n, Y=n, Z=n, dt=0.18, mach=0.1, reynolds=100, ref_length=n,
                   bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann"),
                        cases.BC("lid", 1, 1, 0, 0, "dirichlet", "neumann")])
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    rt, vt, val = cases.bc_arrays(ma, c)
    s0 = np.zeros((ma.total_cells, 4))
    s0[:, 3] = 1.0
    cfg = dict(visc=c.visc, gamma=1.0, dt=c.dt, domain_dt=0.5, pressure_gradient=0.0,
               channel_height=c.Y, max_velocity=c.mach, ref_rho=1.0, tolerance=0.0,
               origin=(0, 0, 0), lengths=(c.X, c.Y, c.Z), gradient_mode=0)
    o = oracle.OracleRun(ma, rt, vt, val, cfg, s0)
    o.run_steps(50)
    s = capi.Solver(ma, rt, vt, val, dict(cfg, renumber=1, precision=capi.FP32_DEVIATION))
    s.set_state(s0)
    s.run(50)
    errs = _field_errors(s.get_state(), o.state)
    print("fp32 vs fp64, 32^3 cavity, 50 steps:", errs)
    assert max(errs.values()) < RUN_TOL, errs


# thousands of steps with IBM, relative L2 per field (measured on the B200 at
# 2,000 steps: u 9.1e-7, v and w 1.1e-5, rho - rho0 8.7e-5; Cd 2.0e-5)
LONG_TOL = {"u": 5e-6, "v": 5e-5, "w": 5e-5, "rho-rho0": 3e-4}


def test_fp32_sphere_channel_2000_steps(plfbs_lib):
    """The 128 x 64 x 64 channel with its 3,217-node sphere (the benchmarked
    configuration), 2,000 steps from the bench's uniform start in both
    precisions: the FP32 deviation form against the FP64 path (itself held to
    the reference's CUDA path at 1e-10 in test_gpu_bench_configs.py), per
    field, and the sphere's drag and lift."""
    import bench
    w, steps = bench.SPHERE, 2000
    pm, c, ma, nodes, s0 = bench.build_channel(w)
    rt, vt, val = cases.bc_arrays(ma, c)
    area = np.pi * w.diam ** 2 / 4
    out = {}
    for prec in (capi.FP64, capi.FP32_DEVIATION):
        s = capi.Solver(ma, rt, vt, val, bench.solver_cfg(c, prec), ibm=bench.ibm_cfg(w, nodes))
        s.set_state(s0)
        st, _ = s.run(steps, history=False)
        assert st["rc"] == 0 and st["steps_done"] == steps
        out[prec] = (s.get_state(), s.body_force(area))
        s.close()
    (q64, (cd64, cl64)), (q32, (cd32, cl32)) = out[capi.FP64], out[capi.FP32_DEVIATION]
    errs = _field_errors(q32[: ma.n_cells], q64[: ma.n_cells])
    cd_err = abs(cd32 - cd64) / abs(cd64)
    print("fp32 vs fp64, 128x64x64 channel, %d steps: %s; Cd %.6f vs %.6f (%.1e), Cl %.2e vs %.2e"
          % (steps, errs, cd32, cd64, cd_err, cl32, cl64))
    assert all(errs[k] < LONG_TOL[k] for k in LONG_TOL), errs
    assert cd_err < 1e-4
