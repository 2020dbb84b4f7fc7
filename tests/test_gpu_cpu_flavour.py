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
