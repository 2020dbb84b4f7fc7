"""Drag and lift over mesh wall faces on the device (plfbs_wall_forces)
against the reference's own post_processing::cylinder_post_processing,
which its GPU driver runs at convergence (Solver_gpu.cu:881-884) and whose
coefficients the golden fixture `converge` holds (`wall_forces`)."""

import numpy as np
import pytest

import golden_cases
from conftest import load_golden
from plfbs import capi, cases

pytestmark = pytest.mark.gpu


def _solver(d, precision=capi.FP64, renumber=0):
    cfg = golden_cases.oracle_cfg(d)
    cfg["renumber"] = renumber
    cfg["precision"] = precision
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    ibm = dict(node_ref=d["nodes"], node_x=d["nodes"], stiffness=cfg["stiffness"],
               radius=cfg["radius"], depth=cfg["depth"], object_nodes=cfg["object_nodes"])
    return capi.Solver(d["ma"], rt, vt, val, cfg, ibm=ibm)


def _walls(d):
    return [i for i, t in enumerate(d["ma"].bc_types) if t == "wall"]


@pytest.mark.parametrize("renumber", [0, 1])
def test_wall_forces_of_the_reference_final_state(plfbs_lib, renumber):
    g = load_golden("converge")
    d = golden_cases.build("converge")
    s = _solver(d, renumber=renumber)
    s.set_state(g["final_state"])
    cd, cl = s.wall_forces(_walls(d))
    ref_cd, ref_cl = g["wall_forces"]
    assert abs(cd - ref_cd) <= 1e-10 * abs(ref_cd)
    assert abs(cl - ref_cl) <= 1e-10 * abs(ref_cl)
    assert s.wall_forces(_walls(d)) == (cd, cl)  # leaves the state as it was


def test_wall_forces_after_a_converged_run(plfbs_lib):
    """The run halts at convergence; the forces still come from fresh gradients."""
    g = load_golden("converge")
    d = golden_cases.build("converge")
    s = _solver(d, renumber=1)
    s.set_state(d["state0"])
    st, _ = s.run(5)
    assert st["converged"] and st["steps_done"] == 1
    cd, cl = s.wall_forces(_walls(d))
    ref_cd, ref_cl = g["wall_forces"]
    assert abs(cd - ref_cd) <= 1e-9 * abs(ref_cd)
    assert abs(cl - ref_cl) <= 1e-9 * abs(ref_cl)
    f32 = _solver(d, precision=capi.FP32_DEVIATION)
    f32.set_state(g["final_state"])
    cd32, cl32 = f32.wall_forces(_walls(d))
    assert abs(cd32 - ref_cd) <= 1e-3 * abs(ref_cd)
    assert abs(cl32 - ref_cl) <= 1e-4 * abs(ref_cl)


def test_wall_forces_rejects_bad_walls(plfbs_lib):
    d = golden_cases.build("channel")
    s = _solver(d)
    s.set_state(d["state0"])
    with pytest.raises(capi.PlfbsError) as e:
        s.wall_forces([d["ma"].n_bc])
    assert e.value.code == capi.ERR_ARG
    inlet = [i for i, t in enumerate(d["ma"].bc_types) if t == "inlet"]  # parabolic: type 9
    with pytest.raises(capi.PlfbsError) as e:
        s.wall_forces(inlet[:1])
    assert e.value.code == capi.ERR_BC
    walls = [i for i, t in enumerate(d["ma"].bc_types) if t == "wall"]
    cd, cl = s.wall_forces(walls)
    assert np.isfinite(cd) and np.isfinite(cl)
