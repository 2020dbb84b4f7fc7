"""Bounded host waits: with a limit far below a batch's run time plfbs_run
returns PLFBS_ERR_TIMEOUT while its 2048 launched steps are still (legitimately)
running; the context answers PLFBS_ERR_TIMEOUT until plfbs_wait sees them end,
then carries on from them to the same state as an uninterrupted run. Nothing
here hangs or faults a GPU: the kernels run to completion, only the host stops
waiting early."""

import numpy as np
import pytest

import golden_cases
from conftest import rel_l2
from plfbs import capi, cases

pytestmark = pytest.mark.gpu


def _solver():
    d = golden_cases.build("cavity")
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    cfg = dict(golden_cases.oracle_cfg(d), tolerance=0.0)
    s = capi.Solver(d["ma"], rt, vt, val, cfg)  # no IBM nodes: deterministic steps
    s.set_state(d["state0"])
    return s


def test_run_times_out_and_the_context_carries_on(plfbs_lib):
    ref = _solver()
    st, _ = ref.run(3000, history=False)
    assert st["steps_done"] == 3000
    want = ref.get_state()
    ref.close()

    s = _solver()
    s.set_timeout(1e-6)
    with pytest.raises(capi.PlfbsError) as e:
        s.run(3000, history=False)
    assert e.value.code == capi.ERR_TIMEOUT
    try:  # still in flight, unless the batch has ended since
        s.get_state()
    except capi.PlfbsError as busy:
        assert busy.code == capi.ERR_TIMEOUT
    assert s.wait(120.0)
    assert s.wait(0.0)  # idle: answers at once
    s.set_timeout(0.0)
    st, _ = s.run(0, history=False)
    assert st["steps_done"] == 2048  # the timed-out batch ran to its end
    st, hist = s.run(3000 - 2048)
    assert st["steps_done"] == 3000 and len(hist) == 3000 - 2048
    got = s.get_state()
    for k in range(4):
        assert rel_l2(got[:, k], want[:, k]) < 1e-12, k
    s.close()
