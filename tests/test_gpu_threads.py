"""Contexts used from several host threads at once (each context single-
threaded, as include/plfbs.h allows): eight threads each create a context on
the same device, capture its step graph, set a state, run and read it back,
all overlapping, and every result is bit for bit the result of the same
solve run alone. A device-wide synchronisation anywhere in those calls would
end another thread's graph capture with an error."""

import threading

import numpy as np
import pytest

import golden_cases
from plfbs import capi, cases

pytestmark = pytest.mark.gpu


def _solve(d, steps, out, k):
    cfg = golden_cases.oracle_cfg(d)
    cfg.update(renumber=k % 3)  # every cell order, built concurrently
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    s = capi.Solver(d["ma"], rt, vt, val, cfg)
    s.set_state(d["state0"])
    st, _ = s.run(steps, history=False)
    out[k] = (st["rc"], s.get_state())
    s.close()


def test_eight_threads_create_and_run_concurrently(plfbs_lib):
    d = golden_cases.build("graded")  # no IBM: every run deterministic
    steps = 40
    want = {}
    for k in range(3):
        _solve(d, steps, want, k)
    for rep in range(3):
        got, errs = {}, []

        def work(k):
            try:
                _solve(d, steps, got, k)
            except Exception as e:  # reported below, with the thread's index
                errs.append((k, repr(e)))

        th = [threading.Thread(target=work, args=(k,)) for k in range(8)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not errs, errs
        for k in range(8):
            assert got[k][0] == 0
            np.testing.assert_array_equal(got[k][1], want[k % 3][1])
