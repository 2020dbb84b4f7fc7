"""Run the reference program (oracle/_ref/plfbs_ref, built from the reference's
own sources by oracle/ref/Makefile) on a synthetic case and load its dumps.

Test infrastructure only: used by make_golden.py to produce the committed
golden fixtures. With <gpu_solver>1</gpu_solver> the reference's CUDA kernels
run serially on the host (oracle/ref/ref_gpu_host.cpp) and PLFBS_REF_DUMP makes
it write .npy arrays; with 0 the reference CPU Solver runs.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "3d-plfbs-gpu_b200"))

from plfbs import cases  # noqa: E402

REF_BIN = os.path.join(REPO, "oracle", "_ref", "plfbs_ref")


def write_restart(out_dir, state):
    """Initial field for <restart_analysis>true</restart_analysis>: the
    "i ,value" text files Solution::import reads (Solution.cpp:987-1064),
    written at full precision. ``state`` is [total_cells, 4] = (u, v, w, rho)."""
    for k, name in enumerate(("u", "v", "w", "rho")):
        with open(os.path.join(out_dir, name + ".txt"), "w") as f:
            f.write("".join("%d ,%.17g\n" % (i, v) for i, v in enumerate(state[:, k])))


def run_reference(workdir, pm, case, nodes=None, init_state=None, dump=True, timeout=600,
                  binary=None, log=None):
    """Write ``pm``/``case`` under ``workdir``, run the reference program (or
    ``binary``, another build of it), return the .npy dumps it wrote. With a
    list ``log``, the console lines of the (last) run are appended to it."""
    binary = binary or REF_BIN
    workdir = os.path.abspath(workdir)
    os.makedirs(workdir, exist_ok=True)
    mesh_dir = os.path.join(workdir, "polyMesh")
    cases.write_polymesh(mesh_dir, pm)
    case.mesh_dir = mesh_dir
    case.output_dir = os.path.join(workdir, "out") + "/"
    if nodes is None:
        nodes = np.zeros((1, 3)) + np.asarray(case.obj_centre)[None, :]
    node_file = os.path.join(workdir, "nodes.txt")
    cases.write_spring_network(node_file, nodes)
    case.obj_nodes_file = node_file
    case.obj_num_nodes = int(nodes.shape[0])
    xml = os.path.join(workdir, "case.xml")
    env = dict(os.environ)
    if init_state is not None:
        steps, restart = case.steps, case.restart
        case.steps, case.restart = 0, False
        cases.write_xml(xml, case)
        subprocess.run([binary, xml], cwd=workdir, env=env, check=True,
                       stdout=subprocess.DEVNULL, timeout=timeout)
        outs = [d for d in glob.glob(os.path.join(workdir, "out", "*")) if os.path.isdir(d)]
        assert len(outs) == 1, outs
        write_restart(outs[0], init_state)
        case.steps, case.restart = steps, True
    cases.write_xml(xml, case)
    dump_dir = os.path.join(workdir, "dump")
    os.makedirs(dump_dir, exist_ok=True)
    if dump:
        env["PLFBS_REF_DUMP"] = dump_dir
    p = subprocess.run([binary, xml], cwd=workdir, env=env, check=True, timeout=timeout,
                       stdout=subprocess.PIPE if log is not None else subprocess.DEVNULL,
                       text=True)
    if log is not None:
        log.extend(p.stdout.splitlines())
    return {os.path.splitext(os.path.basename(p))[0]: np.load(p)
            for p in glob.glob(os.path.join(dump_dir, "*.npy"))}
