"""The CPU-Solver flavour (plfbs_config.flavour = PLFBS_FLAVOUR_CPU_SOLVER)
against the reference CPU Solver itself: fixtures cpu_<case>.npz hold the
final state the reference program writes with <gpu_solver>0</gpu_solver>
(oracle/_ref/plfbs_ref_cpu, run by tests/golden/make_golden.py). Bar: 1e-10
relative L2 per field over the interior cells (the CPU Solver never updates
the ghost cells of the state it outputs)."""

import numpy as np
import pytest

import golden_cases
from conftest import load_golden, rel_l2
from plfbs import capi, cases

pytestmark = pytest.mark.gpu


def _solver(d, renumber):
    cfg = golden_cases.oracle_cfg(d)
    cfg.update(renumber=renumber, flavour=capi.FLAVOUR_CPU_SOLVER)
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    return capi.Solver(d["ma"], rt, vt, val, cfg)


@pytest.mark.parametrize("renumber", [0, 1])
@pytest.mark.parametrize("name", golden_cases.CPU_NAMES)
def test_cpu_flavour_matches_the_cpu_solver(plfbs_lib, name, renumber):
    d = golden_cases.build_cpu(name)
    g = load_golden(name)
    np.testing.assert_array_equal(d["state0"], g["state_init"])
    s = _solver(d, renumber)
    s.set_state(d["state0"])
    st, _ = s.run(int(g["steps"][0]))
    assert st["steps_done"] == int(g["steps"][0])
    C = d["ma"].n_cells
    got, want = s.get_state()[:C], g["final_state"][:C]
    assert np.abs(want - g["state_init"][:C]).max() > 1e-4  # the run moved the field
    for k in range(4):
        assert rel_l2(got[:, k], want[:, k]) < 1e-10, k


def test_gpu_flavour_differs_from_the_cpu_solver(plfbs_lib):
    """Same case, the GPU kernels' tables: the CPU Solver is not what they compute."""
    d = golden_cases.build_cpu("cpu_cavity")
    g = load_golden("cpu_cavity")
    cfg = golden_cases.oracle_cfg(d)
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    s = capi.Solver(d["ma"], rt, vt, val, cfg)
    s.set_state(d["state0"])
    s.run(int(g["steps"][0]))
    C = d["ma"].n_cells
    assert rel_l2(s.get_state()[:C, 0], g["final_state"][:C, 0]) > 1e-6


def _tet_solver(d, flavour):
    c = d["case"]
    cfg = dict(visc=c.visc, gamma=1.0, dt=c.dt, domain_dt=0.5, pressure_gradient=0.0,
               channel_height=c.Y, max_velocity=c.mach, ref_rho=1.0, tolerance=0.0,
               origin=(0, 0, 0), lengths=(c.X, c.Y, c.Z), gradient_mode=capi.GRAD_GREEN_GAUSS,
               renumber=1, flavour=flavour)
    rt, vt, val = cases.bc_arrays(d["ma"], c)
    return capi.Solver(d["ma"], rt, vt, val, cfg)


def test_cpu_flavour_on_20_percent_jittered_tets(plfbs_lib, tmp_path):
    """The unstructured stress mesh at small size (12^3 hexes, nodes jittered
    +-20 %, 10,368 tets, Taylor-Green, Re 400, Green-Gauss): 100 steps against
    the reference CPU Solver run here (1e-10 relative L2), then on to the
    reference's own divergence test, which both fail in the same step."""
    import os

    import refrun
    from conftest import REPO
    binary = os.path.join(REPO, "oracle", "_ref", "plfbs_ref_cpu")
    if not os.path.exists(binary):
        pytest.skip("oracle/_ref/plfbs_ref_cpu not built (needs the reference sources)")
    d = golden_cases.build_tgv_tets(jitter=0.2, steps=100)
    want = refrun.run_reference(str(tmp_path / "r100"), d["pm"], d["case"],
                                init_state=d["state0"], binary=binary)["cpu_final_state"]
    s = _tet_solver(d, capi.FLAVOUR_CPU_SOLVER)
    s.set_state(d["state0"])
    st, _ = s.run(100)
    C = d["ma"].n_cells
    got = s.get_state()[:C]
    for k in range(4):
        assert rel_l2(got[:, k], want[:C, k]) < 1e-10, k
    d400 = golden_cases.build_tgv_tets(jitter=0.2, steps=400)
    log = []
    refrun.run_reference(str(tmp_path / "r400"), d400["pm"], d400["case"],
                         init_state=d400["state0"], binary=binary, dump=False, log=log)
    fail = golden_cases.failure_step(log)  # the reference's loop index t
    assert fail is not None
    st, _ = s.run(400)
    assert st["rc"] == capi.ERR_DIVERGED
    assert st["steps_done"] == fail + 1
    s.close()


def test_gpu_flavour_diverges_on_20_percent_jittered_tets(plfbs_lib):
    """The GPU kernels' tables on the same mesh fail the same test too (the
    reference's GPU path has no tetrahedra to compare with: exactly six
    neighbours, LBFS.cu:1549-1556)."""
    d = golden_cases.build_tgv_tets(jitter=0.2, steps=400)
    s = _tet_solver(d, capi.FLAVOUR_GPU)
    s.set_state(d["state0"])
    st, _ = s.run(400)
    assert st["rc"] == capi.ERR_DIVERGED and 250 < st["steps_done"] < 400
    s.close()
