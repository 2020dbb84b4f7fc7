"""What the trained warm-start network (plfbs/data/warmstart_params.npz) gains
over the plain method, on members of its family it was not trained on: the
first six held-out cases of plfbs/data/warmstart_results.json, taken in order.
The start field's error against the converged field (held-out case 1, Re
137.4: measured 0.053), and the steps the FP32 solver needs to bring the
residual below 1e-5 from the network's start versus from uniform flow
(measured over the six: 66,964 vs 87,199, fewer in each). The evaluation over
all 20 held-out cases down to 1e-6 is in the same file."""

import json
import os

import numpy as np
import pytest

from plfbs import capi, warmstart

pytestmark = pytest.mark.gpu

RESULTS = os.path.join(os.path.dirname(warmstart.__file__), "data", "warmstart_results.json")


def _held_out():
    with open(RESULTS) as f:
        return json.load(f)["held_out"]


def test_start_error_of_a_held_out_case(plfbs_lib):
    case = _held_out()[1]
    ws = warmstart.WarmStarter()
    rec, q_ref = ws.ch.solve(case["re"], case["centre"], capi.FP32_DEVIATION, tol=1e-6,
                             max_steps=80000)
    assert rec["converged"]
    ref = warmstart.to_target(ws.ch, q_ref)
    err_nn = warmstart.rel_l2(ws.predict(case["re"], case["centre"]), ref)
    err_uniform = warmstart.rel_l2(np.zeros_like(ref), ref)
    ws.close()
    assert err_nn < 0.1 * err_uniform
    assert abs(err_nn - case["start_error_nn"]) < 0.01


def test_trained_network_gains_over_uniform_start(plfbs_lib):
    ws = warmstart.WarmStarter()
    cold_steps, warm_steps = [], []
    for case in _held_out()[:6]:
        re, centre = case["re"], case["centre"]
        cold, _ = ws.ch.solve(re, centre, capi.FP32_DEVIATION, tol=1e-5, max_steps=40000)
        warm, _ = ws.ch.solve(re, centre, capi.FP32_DEVIATION, tol=1e-5, max_steps=40000,
                              start=ws.start(re, centre))
        assert cold["converged"] and warm["converged"]
        # FP32 IBM spreading adds in a varying order: the counts move by a few
        assert abs(cold["steps"] - case["fp32"]["steps_to_1e5"]) < 0.02 * cold["steps"]
        assert abs(warm["steps"] - case["fp32_nn"]["steps_to_1e5"]) < 0.02 * warm["steps"]
        cold_steps.append(cold["steps"])
        warm_steps.append(warm["steps"])
    ws.close()
    print("steps to 1e-5, cold:", cold_steps, "warm:", warm_steps)
    assert sum(w < c for w, c in zip(warm_steps, cold_steps)) >= 5
    assert sum(warm_steps) < 0.95 * sum(cold_steps)
