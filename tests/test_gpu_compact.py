"""The compact layout (bitwise-equal face records and cell weight sets
stored once, plfbs_set_layout_compression) against the per-item arrays: the
kernels read the same bits, so a stage's fluxes and whole runs agree bit for
bit (to rounding where several IBM nodes spread into one cell, whose FP64
atomics add in a varying order). A structured box compresses to a handful of
records; a mesh whose records differ everywhere has no compact layout."""

import numpy as np
import pytest

import golden_cases
from plfbs import capi, cases

pytestmark = pytest.mark.gpu


def _box(nx=40, ny=20, nz=20):
    pm = cases.uniform_box(nx, ny, nz, patch_types=["inlet", "outlet", "side", "side", "side",
                                                    "side"])
    c = cases.Case(mesh_dir="", X=nx, Y=ny, Z=nz, dt=0.1, mach=0.05, reynolds=100.0,
                   ref_length=8.0,
                   bcs=[cases.BC("inlet", 1, 1, 0, 0, "dirichlet", "neumann"),
                        cases.BC("outlet", 1, 0, 0, 0, "neumann", "dirichlet"),
                        cases.BC("side", 1, 0, 0, 0, "neumann", "neumann")])
    return cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min), c


def _compare(make, q0, steps, exact):
    out = []
    for on in (0, 1):
        s = make()
        s.set_layout_compression(on)
        s.set_state(q0)
        s.run_stages(1)
        flux = s.face_flux()
        s.run_stages(3)
        _, h = s.run(steps, history=True)
        out.append((flux, s.get_state(), h))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    if exact:
        np.testing.assert_array_equal(out[0][1], out[1][1])
        np.testing.assert_array_equal(out[0][2], out[1][2])
    else:
        np.testing.assert_allclose(out[1][1], out[0][1], rtol=1e-11, atol=1e-14)


@pytest.mark.parametrize("flavour,precision", [(capi.FLAVOUR_GPU, capi.FP64),
                                               (capi.FLAVOUR_CPU_SOLVER, capi.FP64),
                                               (capi.FLAVOUR_GPU, capi.FP32_DEVIATION)])
@pytest.mark.parametrize("renumber", [0, 1])
def test_compact_box_is_bitwise_equal(plfbs_lib, renumber, flavour, precision):
    ma, c = _box()
    rt, vt, val = cases.bc_arrays(ma, c)
    cfg = dict(visc=c.visc, dt=c.dt, max_velocity=c.mach, channel_height=c.Y,
               lengths=(c.X, c.Y, c.Z), renumber=renumber, flavour=flavour,
               pressure_gradient=1e-5, precision=precision)
    ibm = None
    # IBM on the FP64 GPU flavour only: its FP64 atomics reorder to rounding
    # (compared to 1e-11); the FP32 and CPU-flavour runs compare bit for bit
    if flavour == capi.FLAVOUR_GPU and precision == capi.FP64:
        nodes = cases.fibonacci_sphere(150, 4.0, (12.0, 10.0, 10.0))
        ibm = dict(node_ref=nodes, stiffness=0.5, radius=4.0, depth=8.0, object_nodes=len(nodes))
    rng = np.random.default_rng(9)
    q0 = np.zeros((ma.total_cells, 4))
    q0[:, 0] = 0.05 + 0.005 * rng.standard_normal(ma.total_cells)
    q0[:, 1:3] = 0.002 * rng.standard_normal((ma.total_cells, 2))
    q0[:, 3] = 1.0 + 0.001 * rng.standard_normal(ma.total_cells)
    probe = capi.Solver(ma, rt, vt, val, cfg, ibm=ibm)
    nf, nc = probe.layout()["compact"]
    assert 0 < nf <= 64 and 0 < nc <= 64, (nf, nc)  # a structured box repeats its geometry
    probe.close()
    _compare(lambda: capi.Solver(ma, rt, vt, val, cfg, ibm=ibm), q0, 10, exact=ibm is None)


@pytest.mark.parametrize("name", golden_cases.NAMES)
def test_compact_golden_meshes(plfbs_lib, name):
    d = golden_cases.build(name)
    cfg = golden_cases.oracle_cfg(d)
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    ibm = dict(node_ref=d["nodes"], node_x=d["nodes"], stiffness=cfg["stiffness"],
               radius=cfg["radius"], depth=cfg["depth"], object_nodes=cfg["object_nodes"])
    make = lambda: capi.Solver(d["ma"], rt, vt, val, cfg, ibm=ibm)  # noqa: E731
    s = make()
    if s.layout()["compact"] == (0, 0):
        with pytest.raises(capi.PlfbsError) as e:
            s.set_layout_compression(1)
        assert e.value.code == capi.ERR_ARG
        return
    _compare(make, d["state0"], 3, exact=len(d["nodes"]) <= 1)


def test_tets_have_no_compact_layout(plfbs_lib):
    pm = cases.jittered_tet_box(6, jitter=0.1, seed=4, patch_types=["wall"] * 6)
    c = cases.Case(mesh_dir="", X=6, Y=6, Z=6, dt=0.05, mach=0.05, reynolds=100.0,
                   ref_length=6.0, bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann")])
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    rt, vt, val = cases.bc_arrays(ma, c)
    s = capi.Solver(ma, rt, vt, val, dict(visc=c.visc, dt=c.dt, max_velocity=c.mach,
                                          lengths=(6, 6, 6)))
    assert s.layout()["compact"] == (0, 0)
    with pytest.raises(capi.PlfbsError) as e:
        s.set_layout_compression(1)
    assert e.value.code == capi.ERR_ARG
    s.set_layout_compression(0)
