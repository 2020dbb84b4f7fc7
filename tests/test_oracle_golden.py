"""The oracle and the case builder against the reference's own outputs.

Fixtures (tests/golden/*.npz) are dumps of the reference's kernels compiled
from its sources and run on the host (oracle/ref/, make_golden.py). No GPU.
"""

import numpy as np
import pytest

import golden_cases
import oracle
from conftest import load_golden, rel_err
from plfbs import cases

NAMES = golden_cases.NAMES


@pytest.mark.parametrize("name", NAMES)
def test_mesh_arrays_bit_exact(name):
    """cases.mesh_arrays reproduces unstructured_mesh's geometry bit for bit."""
    g = load_golden(name)
    ma = golden_cases.build(name)["ma"]
    C, F, Fi, B, T = (int(x) for x in g["sizes"])
    assert (ma.n_cells, ma.n_faces, ma.n_internal, ma.n_bc) == (C, F, Fi, B)
    for key in ("owner", "neighbour", "face_area", "face_normal", "face_centroid",
                "streaming_dt", "cell_volume", "cell_centroid"):
        np.testing.assert_array_equal(getattr(ma, key), g[key], err_msg=key)
    np.testing.assert_array_equal(ma.stencil_cells.reshape(C, 6), g["stencil"])


@pytest.mark.parametrize("name", NAMES)
def test_bc_arrays(name):
    d = golden_cases.build(name)
    g = load_golden(name)
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    np.testing.assert_array_equal(rt, g["bc_rho_type"])
    np.testing.assert_array_equal(vt, g["bc_vel_type"])
    np.testing.assert_array_equal(val, g["bc_value"])
    np.testing.assert_array_equal(d["state0"], g["state_init"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_ls_weights_bit_exact(name):
    d = golden_cases.build(name)
    g = load_golden(name)
    mode = golden_cases.oracle_cfg(d)["gradient_mode"]
    lhs, rhs = oracle.ls_weights(d["ma"], mode)
    np.testing.assert_array_equal(lhs, g["lhs_inv"])
    np.testing.assert_array_equal(rhs.reshape(-1, 6, 3), g["rhs_w"])


def _oracle(name):
    d = golden_cases.build(name)
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    return d, oracle.OracleRun(d["ma"], rt, vt, val, golden_cases.oracle_cfg(d), d["state0"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_first_stage(name):
    """One RK stage: ghost states, gradients (ghosts included), face fluxes,
    residuals and the stage state against the reference kernels."""
    d, o = _oracle(name)
    g = load_golden(name)
    C = d["ma"].n_cells
    o.run_stages(1)
    np.testing.assert_array_equal(o.state[C:], g["s0_state_bc"][C:])  # ghost states
    assert rel_err(o.grad, g["s0_grad"]) < 1e-14
    assert rel_err(o.face_flux, g["s0_face_flux"]) < 1e-14
    assert rel_err(o.residual, g["s0_residual"]) < 1e-13
    assert rel_err(o.state[:C], g["s0_state_rk"][:C]) < 1e-15
    assert rel_err(o.force, g["s0_force"]) < 1e-14
    assert rel_err(o.node_x, g["s0_nodes"][:, 0:3]) < 1e-15
    assert rel_err(o.node_vel, g["s0_nodes"][:, 3:6]) < 1e-14
    assert rel_err(o.node_force, g["s0_nodes"][:, 6:9]) < 1e-13


@pytest.mark.parametrize("name", NAMES)
def test_oracle_full_run(name):
    """All steps, stopping on convergence exactly as the reference does."""
    d, o = _oracle(name)
    g = load_golden(name)
    steps = o.run_steps(d["case"].steps, stop_on_convergence=True)
    assert steps == int(g["steps_done"][0])
    assert rel_err(o.state, g["final_state"]) < 1e-14
    assert rel_err(o.t1, g["final_t1"][: d["ma"].n_cells]) < 1e-14
    assert rel_err(o.history, g["history"]) < 1e-12
    assert rel_err(o.node_x, g["final_nodes"][:, 0:3]) < 1e-15


@pytest.mark.parametrize("name", golden_cases.CPU_NAMES)
def test_oracle_cpu_flavour_matches_the_cpu_solver(name):
    """The oracle's CPU-Solver restatement (flavour 1) against the reference CPU
    Solver's own final state (tests/golden/cpu_*.npz): 1e-10 per field."""
    d = golden_cases.build_cpu(name)
    g = load_golden(name)
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    cfg = dict(golden_cases.oracle_cfg(d), flavour=1)
    o = oracle.OracleRun(d["ma"], rt, vt, val, cfg, d["state0"])
    o.run_steps(int(g["steps"][0]))
    C = d["ma"].n_cells
    for k in range(4):
        a, b = o.state[:C, k], g["final_state"][:C, k]
        assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b), k
