"""Checkpoint/restart and warm start through the C ABI.

A checkpoint taken at a step boundary and loaded into a fresh context built
from the same inputs must continue the run bit for bit where the step is
deterministic (no two IBM nodes spreading into one cell), and to rounding
where FP64 atomics from several nodes meet. plfbs_warm_start seeds the RK
accumulators with the conserved variables, so restarting from a solution
continues it; plfbs_set_state keeps the reference's velocity seeding.
"""

import numpy as np
import pytest

import golden_cases
from conftest import rel_err
from plfbs import capi, cases

pytestmark = pytest.mark.gpu


def _solver(d, precision=capi.FP64, renumber=1):
    cfg = golden_cases.oracle_cfg(d)
    cfg["renumber"] = renumber
    cfg["precision"] = precision
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    ibm = dict(node_ref=d["nodes"], node_x=d["nodes"], stiffness=cfg["stiffness"],
               radius=cfg["radius"], depth=cfg["depth"], object_nodes=cfg["object_nodes"])
    return capi.Solver(d["ma"], rt, vt, val, cfg, ibm=ibm)


def _resume(name, precision):
    d = golden_cases.build(name)
    a = _solver(d, precision)
    a.set_state(d["state0"])
    _, ha = a.run(6, history=True)
    b = _solver(d, precision)
    b.set_state(d["state0"])
    b.run(3)
    image = b.checkpoint()
    b.close()
    c = _solver(d, precision)
    c.restore(image)
    _, hc = c.run(3, history=True)
    return a, c, ha, hc


@pytest.mark.parametrize("precision", [capi.FP64, capi.FP32_DEVIATION])
def test_resume_is_bitwise(plfbs_lib, precision):
    """graded: one IBM node, so every cell receives at most one atomic add."""
    a, c, ha, hc = _resume("graded", precision)
    np.testing.assert_array_equal(a.get_state(), c.get_state())
    np.testing.assert_array_equal(ha[3:], hc)
    xa, va, fa = a.nodes()
    xc, vc, fc = c.nodes()
    np.testing.assert_array_equal(xa, xc)
    np.testing.assert_array_equal(fa, fc)


def test_resume_with_ibm_sphere(plfbs_lib):
    """channel: 34 nodes whose spreading can meet in a cell (atomic order)."""
    a, c, ha, hc = _resume("channel", capi.FP64)
    assert rel_err(c.get_state(), a.get_state()) < 1e-12
    np.testing.assert_allclose(hc[:, 1:], ha[3:, 1:], rtol=1e-9, atol=0)
    np.testing.assert_array_equal(hc[:, 0], ha[3:, 0])  # step numbers continue


def test_checkpoint_rejects_other_mesh_and_precision(plfbs_lib):
    g = golden_cases.build("graded")
    a = _solver(g)
    a.set_state(g["state0"])
    image = a.checkpoint()
    other = _solver(golden_cases.build("cavity"))
    with pytest.raises(capi.PlfbsError) as e:
        other.restore(image)
    assert e.value.code == capi.ERR_MESH
    f32 = _solver(g, capi.FP32_DEVIATION)
    with pytest.raises(capi.PlfbsError) as e:
        f32.restore(image)
    assert e.value.code == capi.ERR_ARG
    with pytest.raises(capi.PlfbsError):
        a.restore(image[:100])


def test_warm_start_continues_a_run(plfbs_lib):
    """Restarting from get_state + node positions with conserved seeding
    reproduces the continuing run to rounding; the reference's velocity seeding
    (plfbs_set_state) perturbs it by about |rho - 1|."""
    d = golden_cases.build("channel")
    a = _solver(d)
    a.set_state(d["state0"])
    a.run(20)
    q = a.get_state()
    x = a.nodes()[0]
    assert np.abs(q[:, 3] - 1.0).max() > 1e-6  # density has moved off 1
    a.run(1)
    ref = a.get_state()
    w = _solver(d)
    w.warm_start(q, x)
    w.run(1)
    s = _solver(d)
    s.set_state(q)
    s.run(1)
    # nodes of `s` start at the reference positions; compare fluid only
    err_warm = rel_err(w.get_state(), ref)
    err_quirk = rel_err(s.get_state(), ref)
    assert err_warm < 1e-10
    assert err_quirk > 100 * err_warm
