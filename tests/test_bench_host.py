"""bench.py's timing of the reference's own CUDA path (reference_gpu): the
median time between its progress lines, over the steps between them, with a
slow first interval (setup-like) left out; and a failed run reported as a
reason instead of a number. A stand-in program prints the progress lines."""

import stat
import sys

import pytest

from conftest import REPO
from plfbs import cases

sys.path.insert(0, REPO)
import bench  # noqa: E402

STAND_IN = """#!/bin/bash
echo "Running Solver"
for i in 1 2 3 4 5 6; do
  echo "time t=$i error e =0.1 delta_t:0.2"
  echo "drag: 0"
  if [ $i -eq 1 ]; then sleep 0.5; else sleep 0.15; fi
done
exit %d
"""


def _case():
    pm = cases.uniform_box(4, 4, 4)
    c = cases.Case(mesh_dir="", X=4, Y=4, Z=4, dt=0.2, mach=0.05, reynolds=100, ref_length=4.0,
                   bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann")])
    return pm, c, cases.fibonacci_sphere(4, 1.0, (2.0, 2.0, 2.0))


@pytest.mark.parametrize("rc", [0, 1])
def test_reference_gpu_timing_from_progress_lines(tmp_path, monkeypatch, rc):
    exe = tmp_path / "stand_in.sh"
    exe.write_text(STAND_IN % rc)
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    monkeypatch.setattr(bench, "REF_GPU_BIN", str(exe))
    pm, c, nodes = _case()
    steps_before = c.steps
    value, sample = bench.reference_gpu_throughput(pm, c, nodes, steps=601, every=100)
    assert c.steps == steps_before  # the caller's case is left as it was
    if rc:
        assert value is None and "exited with 1" in sample
    else:
        per_step = pm.n_cells / value / 1e6  # seconds
        assert 0.0014 < per_step < 0.0025, per_step  # 0.15 s per 100 steps; the 0.5 s one dropped
        assert "median of 5 intervals" in sample


def test_clean_intervals_leave_out_the_text_output():
    """A progress line followed by a decade output: the interval to the next
    line starts at the output's end marker; the CPU Solver's last interval
    ends at "out of time" after its last step."""
    ev = [(0.0, "line"), (3.0, "out"), (5.0, "line"), (7.0, "line"), (8.0, "out"), (9.5, "end")]
    # lines after steps 1, 3, 5 (output_step 2), 7 steps (t = 0 .. 6)
    iv = bench.clean_intervals(ev, 2, 7)
    assert iv == [(2.0, 2), (2.0, 2), (1.5, 1)]
    # a run that never printed its end gives no interval after its last line
    assert bench.clean_intervals(ev[:3], 2, 7) == [(2.0, 2)]


def test_aggregate_of_concurrent_instances():
    cells = 1_000_000
    # all three stepping at once (common instant 2.5): the sum of their rates
    spans = [(10.0, (0.0, 10.0)), (20.0, (2.5, 22.5)), (10.0, (1.0, 11.0))]
    v, how = bench.aggregate(spans, cells)
    assert abs(v - (0.1 + 0.05 + 0.1)) < 1e-12 and "sum" in how
    # staggered: total cell-updates over the whole span, a lower bound
    spans = [(10.0, (0.0, 10.0)), (10.0, (20.0, 30.0))]
    v, how = bench.aggregate(spans, cells)
    assert abs(v - 2 * cells / 30.0 / 1e6) < 1e-12 and "span" in how
