"""The TMA-staged FP64 flux kernel (plfbs_set_flux_kernel(ctx, 1)) against the
per-thread one: the same arithmetic on the same data, so the fluxes of a
stage agree bit for bit, on the golden meshes and on a box of many face
tiles. Whole runs agree bit for bit where at most one IBM node spreads into
a cell; with several, the order of their FP64 atomic additions varies from
run to run (with either kernel) and the runs agree to rounding."""

import numpy as np
import pytest

import golden_cases
from plfbs import capi, cases

pytestmark = pytest.mark.gpu


def _solver(d, renumber, precision=capi.FP64):
    cfg = golden_cases.oracle_cfg(d)
    cfg.update(renumber=renumber, precision=precision)
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    ibm = dict(node_ref=d["nodes"], node_x=d["nodes"], stiffness=cfg["stiffness"],
               radius=cfg["radius"], depth=cfg["depth"], object_nodes=cfg["object_nodes"])
    return capi.Solver(d["ma"], rt, vt, val, cfg, ibm=ibm)


@pytest.mark.parametrize("renumber", [0, 1])
@pytest.mark.parametrize("name", golden_cases.NAMES)
def test_tma_flux_is_bitwise_equal(plfbs_lib, name, renumber):
    d = golden_cases.build(name)
    out = []
    for kind in (0, 1):
        s = _solver(d, renumber)
        s.set_flux_kernel(kind)
        s.set_state(d["state0"])
        s.run_stages(1)
        flux = s.face_flux()
        s.run_stages(3)
        st, h = s.run(5, history=True)
        out.append((flux, s.get_state(), h))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    if len(d["nodes"]) <= 1:
        np.testing.assert_array_equal(out[0][1], out[1][1])
        np.testing.assert_array_equal(out[0][2], out[1][2])
    else:
        np.testing.assert_allclose(out[1][1], out[0][1], rtol=1e-11, atol=1e-14)
        np.testing.assert_allclose(out[1][2][:, 1:], out[0][2][:, 1:], rtol=1e-9, atol=0)


def test_tma_flux_on_many_tiles(plfbs_lib):
    pm = cases.uniform_box(48, 24, 24, patch_types=["inlet", "outlet", "side", "side", "side",
                                                    "side"])
    c = cases.Case(mesh_dir="", X=48, Y=24, Z=24, dt=0.1, mach=0.05, reynolds=100.0,
                   ref_length=8.0,
                   bcs=[cases.BC("inlet", 1, 1, 0, 0, "dirichlet", "neumann"),
                        cases.BC("outlet", 1, 0, 0, 0, "neumann", "dirichlet"),
                        cases.BC("side", 1, 0, 0, 0, "neumann", "neumann")])
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    rt, vt, val = cases.bc_arrays(ma, c)
    nodes = cases.fibonacci_sphere(200, 4.0, (16.0, 12.0, 12.0))
    cfg = dict(visc=c.visc, dt=c.dt, max_velocity=c.mach, channel_height=c.Y,
               lengths=(c.X, c.Y, c.Z), renumber=1)
    ibm = dict(node_ref=nodes, stiffness=0.5, radius=4.0, depth=8.0, object_nodes=len(nodes))
    rng = np.random.default_rng(7)
    q0 = np.zeros((ma.total_cells, 4))
    q0[:, 0] = 0.05 + 0.01 * rng.standard_normal(ma.total_cells)
    q0[:, 1:3] = 0.005 * rng.standard_normal((ma.total_cells, 2))
    q0[:, 3] = 1.0 + 0.001 * rng.standard_normal(ma.total_cells)
    res = []
    for kind in (0, 1):
        s = capi.Solver(ma, rt, vt, val, cfg, ibm=ibm)
        s.set_flux_kernel(kind)
        s.set_state(q0)
        s.run_stages(1)
        flux = s.face_flux()
        s.run_stages(3)
        _, h = s.run(20, history=True)
        res.append((flux, s.get_state(), h))
    assert ma.n_internal > 100 * 128
    np.testing.assert_array_equal(res[0][0], res[1][0])
    np.testing.assert_allclose(res[1][1], res[0][1], rtol=1e-11, atol=1e-14)
    np.testing.assert_allclose(res[1][2][:, 1:], res[0][2][:, 1:], rtol=1e-9, atol=0)


def test_tma_flux_needs_fp64(plfbs_lib):
    d = golden_cases.build("channel")
    s = _solver(d, 0, capi.FP32_DEVIATION)
    with pytest.raises(capi.PlfbsError) as e:
        s.set_flux_kernel(1)
    assert e.value.code == capi.ERR_ARG
    s.set_flux_kernel(0)
    with pytest.raises(capi.PlfbsError):
        _solver(d, 0).set_flux_kernel(2)
