"""Regenerate the golden fixtures tests/golden/<case>.npz from the reference.

    make -C oracle/ref REF=<reference checkout>/src && python tests/golden/make_golden.py

Runs oracle/_ref/plfbs_ref (the reference program, built from its own
sources; its CUDA kernels execute serially on the host) on each case of
golden_cases.py and keeps the dumps the tests compare against: the reference's
pre-processed mesh arrays and least-squares weights, the ghost states,
gradients, face fluxes, residuals and state after the first RK stage, the body
force and Lagrangian nodes after the first IBM update, and the state, RK
accumulator, residual history and nodes after the last step, and (for a run
that converges) the wall drag and lift coefficients of cylinder_post_processing.

The CPU-Solver cases (golden_cases.CPU_NAMES) run oracle/_ref/plfbs_ref_cpu,
the same program with <gpu_solver>0</gpu_solver> whose final state
ref_cpu_dump.cpp writes losslessly; their fixtures cpu_<case>.npz hold the
initial and final states.

    python tests/golden/make_golden.py long

writes the full-length lid-driven cavity fixtures instead (golden_cases
build_cavity32: 32^3, Re 100, 2,000 steps from rest; about ten minutes of
CPU): cavity32.npz from the reference's GPU kernels run serially on the host
(final state, residual history, steps) and cpu_cavity32.npz from the
reference CPU Solver (final state).
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import golden_cases  # noqa: E402
import refrun  # noqa: E402

KEEP = ("sizes", "owner", "neighbour", "stencil", "face_area", "streaming_dt", "face_normal",
        "face_centroid", "cell_volume", "cell_centroid", "lhs_inv", "rhs_w", "bc_value",
        "bc_rho_type", "bc_vel_type", "state_init", "params", "s0_force", "s0_nodes",
        "s0_state_bc", "s0_grad", "s0_face_flux", "s0_residual", "s0_state_rk",
        "final_state", "final_t1", "history", "steps_done", "final_nodes", "wall_forces")


CPU_BIN = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref", "plfbs_ref_cpu")


def main():
    tmp = tempfile.mkdtemp(prefix="plfbs_golden_")
    try:
        for name in golden_cases.CPU_NAMES:
            d = golden_cases.build_cpu(name)
            dumps = refrun.run_reference(os.path.join(tmp, name), d["pm"], d["case"],
                                         init_state=d["state0"], binary=CPU_BIN)
            out = dict(state_init=d["state0"], final_state=dumps["cpu_final_state"],
                       steps=np.array([d["case"].steps], np.int32))
            path = os.path.join(HERE, name + ".npz")
            np.savez_compressed(path, **out)
            print("%-11s %7d bytes  steps=%d" % (name, os.path.getsize(path), d["case"].steps))
        for name in golden_cases.NAMES:
            d = golden_cases.build(name)
            dumps = refrun.run_reference(os.path.join(tmp, name), d["pm"], d["case"],
                                         nodes=d["nodes"], init_state=d["state0"])
            out = {k: dumps[k] for k in KEEP}
            path = os.path.join(HERE, name + ".npz")
            np.savez_compressed(path, **out)
            print("%-9s %7d bytes  steps_done=%d" % (name, os.path.getsize(path),
                                                     int(out["steps_done"][0])))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main_long():
    tmp = tempfile.mkdtemp(prefix="plfbs_golden_")
    try:
        d = golden_cases.build_cavity32()
        dumps = refrun.run_reference(os.path.join(tmp, "cavity32"), d["pm"], d["case"],
                                     init_state=d["state0"], timeout=3600)
        out = {k: dumps[k] for k in ("final_state", "history", "steps_done")}
        np.savez_compressed(os.path.join(HERE, "cavity32.npz"), **out)
        d = golden_cases.build_cavity32(cpu_solver=True)
        dumps = refrun.run_reference(os.path.join(tmp, "cpu_cavity32"), d["pm"], d["case"],
                                     init_state=d["state0"], binary=CPU_BIN, timeout=3600)
        np.savez_compressed(os.path.join(HERE, "cpu_cavity32.npz"),
                            final_state=dumps["cpu_final_state"],
                            steps=np.array([d["case"].steps], np.int32))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "long":
        main_long()
    else:
        main()
