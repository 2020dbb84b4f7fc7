"""The drop-in: the reference program itself, with its GPU solver (or its CPU
Solver) replaced by the shims in 3d-plfbs-gpu_b200/shim over libplfbs, against
the golden dumps of the reference's own kernels (or of its CPU Solver). Needs
oracle/_ref/plfbs_ref_b200 and plfbs_ref_cpu_b200 (built from the reference
sources by `make -C oracle/ref integration`); skipped without them."""

import glob
import json
import os

import numpy as np
import pytest

import golden_cases
import refrun
from conftest import REPO, load_golden, rel_l2

pytestmark = pytest.mark.gpu

BIN = os.path.join(REPO, "oracle", "_ref", "plfbs_ref_b200")
BIN_CPU = os.path.join(REPO, "oracle", "_ref", "plfbs_ref_cpu_b200")


def _check_run_log(tmp_path):
    """The shim's JSON-lines run log: one record per output step, the exit last."""
    paths = glob.glob(os.path.join(str(tmp_path), "out", "*", "run.jsonl"))
    assert len(paths) == 1, paths
    recs = [json.loads(line) for line in open(paths[0]) if line.strip()]
    assert recs and recs[-1]["exit"] in ("converged", "out_of_time", "diverged")
    assert all("max_error" in r for r in recs[:-1])


@pytest.mark.parametrize("name", ["cavity", "channel", "converge"])
def test_reference_program_with_plfbs(tmp_path, name):
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/plfbs_ref_b200 not built (needs the reference sources)")
    d = golden_cases.build(name)
    g = load_golden(name)
    refrun.run_reference(str(tmp_path), d["pm"], d["case"], nodes=d["nodes"],
                         init_state=d["state0"], dump=False, binary=BIN)
    paths = glob.glob(os.path.join(str(tmp_path), "out", "*", "state.bin"))
    assert len(paths) == 1, paths
    T = d["ma"].total_cells
    raw = np.fromfile(paths[0], dtype=np.float64).reshape(4, T)  # rho, u, v, w
    state = np.stack([raw[1], raw[2], raw[3], raw[0]], axis=1)
    for k in range(4):
        assert rel_l2(state[:, k], g["final_state"][:, k]) < 1e-10, k
    _check_run_log(tmp_path)
    # the reference's 6-significant-digit text output agrees too on interior
    # cells (after a converged exit the host re-applies its CPU boundary update
    # to the ghosts before writing, Solver_gpu.cu:882, as the reference does)
    C = d["ma"].n_cells
    u_txt = glob.glob(os.path.join(str(tmp_path), "out", "*", "u.txt"))[0]
    u = np.loadtxt(u_txt, delimiter=",")[:, 1]
    np.testing.assert_allclose(u[:C], g["final_state"][:C, 0], rtol=1e-5, atol=1e-9)


@pytest.mark.parametrize("name", golden_cases.CPU_NAMES)
def test_reference_program_with_plfbs_cpu_solver(tmp_path, name):
    """<gpu_solver>0</gpu_solver>: program.cpp calls Solver::General_Purpose_Solver_mk_i,
    here the CPU shim over the CPU-Solver flavour."""
    if not os.path.exists(BIN_CPU):
        pytest.skip("oracle/_ref/plfbs_ref_cpu_b200 not built (needs the reference sources)")
    d = golden_cases.build_cpu(name)
    g = load_golden(name)
    refrun.run_reference(str(tmp_path), d["pm"], d["case"], init_state=d["state0"], dump=False,
                         binary=BIN_CPU)
    paths = glob.glob(os.path.join(str(tmp_path), "out", "*", "state.bin"))
    assert len(paths) == 1, paths
    T, C = d["ma"].total_cells, d["ma"].n_cells
    raw = np.fromfile(paths[0], dtype=np.float64).reshape(4, T)  # rho, u, v, w
    state = np.stack([raw[1], raw[2], raw[3], raw[0]], axis=1)
    for k in range(4):
        assert rel_l2(state[:C, k], g["final_state"][:C, k]) < 1e-10, k
    _check_run_log(tmp_path)
    u_txt = glob.glob(os.path.join(str(tmp_path), "out", "*", "u.txt"))[0]
    u = np.loadtxt(u_txt, delimiter=",")[:, 1]
    np.testing.assert_allclose(u[:C], g["final_state"][:C, 0], rtol=1e-5, atol=1e-9)
