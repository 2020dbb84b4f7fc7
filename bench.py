#!/usr/bin/env python
"""Throughput of the LBFS explicit time step on B200 (one JSON line on rank 0).

Workload: the sphere-in-channel case — a 128 x 64 x 64 uniform hex channel
(524,288 cells, 1,593,344 faces) with an immersed sphere of diameter 16 cells
at (32, 32, 32) carried by 3,217 Fibonacci-lattice nodes; inlet u = 0.05
(Dirichlet velocity, Neumann density), outlet Neumann velocity with rho = 1,
side walls Neumann in velocity and density (the GPU path has no slip type);
Re = 100 on the diameter (nu = 0.008), RK dt 0.2, FP64. Synthetic, seeded
inputs; uniform-flow start.

A step is one full time step: the IBM update and 4 RK stages over all cells
and faces. `value` is device throughput in Mcell-updates/s (cells x steps /
time, summed over ranks, max time over ranks; `per_rk_stage` is the same
rate per RK stage, 4 x value) with everything resident in
HBM; the working set (~0.5 GB) exceeds the 126 MB L2, so no flush is needed
between steps. `e2e` times the whole drop-in call through the C ABI from host
buffers: create (mesh upload, least-squares weights, layout), set_state,
run, the per-step residual history read-back, get_state and destroy.

--impl reference times the reference's own CPU Solver (oracle/_ref, built
from the reference sources) on the same mesh and boundary conditions.
`reference_gpu` (rank 0, one GPU, FP64) is the reference's own CUDA path
(Solver_gpu.cu built for sm_100a) timed on the same case, outside the timed
region: the reference-kernel figure beside `value`.
"""

from __future__ import annotations

import argparse
import faulthandler
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "3d-plfbs-gpu_b200"))

from plfbs import cases  # noqa: E402

METRIC = "Mcell-updates/s"
E2E_REPS = 3  # end-to-end repetitions (the median is reported)
WORKLOAD = "sphere_channel_128x64x64_ibm3217_fp64"
NX, NY, NZ = 128, 64, 64
DIAM, CENTRE, NNODES = 16.0, (32.0, 32.0, 32.0), 3217
U, RE, DT, STIFFNESS = 0.05, 100.0, 0.2, 0.5
KERNELS_PER_STEP = 14  # ibm + 4 x (gradient, flux, update) + finish

# Algorithmic bytes per launch (FP64, perfect reuse): per face the geometry
# (normal, area, streaming dt, owner/neighbour offsets: 72 B) and the flux
# write (32 B); per cell the state (32 B), gradients (96 B), centroid and
# volume (32 B) read once. gradient: state + 6 weights/indices + gradient
# write; update: 6 face fluxes, indices, t0, t1 read+write, state write.
def algorithmic_bytes(C, F, B, fp32=False):
    if fp32:  # the same traffic with 4-byte values (indices stay 4 bytes)
        return {"flux": 56 * F + 80 * C, "gradient": 160 * C, "update": 196 * C}
    return {"flux": 104 * F + 160 * C,
            "gradient": 296 * C,
            "update": 344 * C}


def build_case():
    pm = cases.uniform_box(NX, NY, NZ, patch_types=["inlet", "outlet", "side", "side", "side",
                                                    "side"])
    c = cases.Case(mesh_dir="", X=NX, Y=NY, Z=NZ, dt=DT, mach=U, reynolds=RE, ref_length=DIAM,
                   tolerance=0.0, obj_radius=DIAM / 2, obj_depth=DIAM, obj_stiffness=STIFFNESS,
                   obj_centre=CENTRE,
                   bcs=[cases.BC("inlet", 1, 1, 0, 0, "dirichlet", "neumann"),
                        cases.BC("outlet", 1, 0, 0, 0, "neumann", "dirichlet"),
                        cases.BC("side", 1, 0, 0, 0, "neumann", "neumann")])
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    nodes = cases.fibonacci_sphere(NNODES, DIAM / 2, CENTRE)
    state0 = np.zeros((ma.total_cells, 4))
    state0[:, 0] = U
    state0[:, 3] = 1.0
    return pm, c, ma, nodes, state0


def solver_cfg(c, precision=0, renumber=0):
    return dict(visc=c.visc, gamma=1.0, dt=c.dt, domain_dt=0.5, max_velocity=c.mach,
                ref_rho=1.0, tolerance=0.0, pressure_gradient=0.0, channel_height=c.Y,
                origin=(0.0, 0.0, 0.0), lengths=(c.X, c.Y, c.Z), gradient_mode=0,
                renumber=renumber, precision=precision)


def ibm_cfg(nodes):
    return dict(node_ref=nodes, stiffness=STIFFNESS, radius=DIAM / 2, depth=DIAM,
                object_nodes=len(nodes))


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.01)

    def __enter__(self):
        if self.nv:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self.nv:
            self.t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def load_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(kernel, workload):
    """ncu DRAM bytes per launch of `kernel` on `workload`, committed under
    profiles/traffic.json by the profiling recipe (null when absent)."""
    try:
        with open(os.path.join(REPO, "profiles", "traffic.json")) as f:
            t = json.load(f)
        return t.get(workload, {}).get(kernel)
    except Exception:
        return None


# ---------------------------------------------------------------------------
# reference arm: the reference's CPU Solver (serial) on the same case
# ---------------------------------------------------------------------------

REF_BIN = os.path.join(REPO, "oracle", "_ref", "plfbs_ref")


def _run_ref_cpu(workdir, pm, c, nodes, steps, mesh_dir=None, progress=None, limit=1200):
    import shutil
    c.steps = steps
    c.gpu_solver = 0
    c.output_dir = os.path.join(workdir, "out") + "/"
    if os.path.isdir(os.path.join(workdir, "out")):
        shutil.rmtree(os.path.join(workdir, "out"))
    node_file = os.path.join(workdir, "nodes.txt")
    if not os.path.exists(node_file):
        cases.write_spring_network(node_file, nodes)
    c.obj_nodes_file = node_file
    c.obj_num_nodes = len(nodes)
    c.mesh_dir = mesh_dir or os.path.join(workdir, "polyMesh")
    xml = os.path.join(workdir, "case.xml")
    cases.write_xml(xml, c)
    # the time from the program's "Running Solver" line (printed right before
    # it calls the solver, program.cpp:106) to its exit: the mesh import and
    # the rest of the setup before it are left out
    p = subprocess.Popen([REF_BIN, xml], cwd=workdir, stdout=subprocess.PIPE,
                         stderr=subprocess.DEVNULL, text=True)
    timer = threading.Timer(limit, p.kill)  # this process only
    timer.start()
    t_solver = None
    stamps = []  # arrivals of its progress lines ("time t=", Solver.cpp:501-508)
    try:
        for line in p.stdout:
            now = time.perf_counter()
            if t_solver is None and line.startswith("Running Solver"):
                t_solver = now
            elif line.startswith("time t="):
                stamps.append(now)
        rc = p.wait()
    finally:
        timer.cancel()
    t_end = time.perf_counter()
    if rc != 0 or t_solver is None:
        raise subprocess.CalledProcessError(rc, REF_BIN)
    if progress is not None:
        progress.extend(stamps)
    return t_end - t_solver


def reference_cpu_throughput(pm, c, nodes, sample_steps=1):
    """Mcell-updates/s of the reference CPU Solver: the solver's time in a run
    of `sample_steps` steps minus that in a 0-step run (its own setup and the
    final output), each timed from the program's "Running Solver" line."""
    if not os.path.exists(REF_BIN):
        return None, "oracle/_ref/plfbs_ref not built"
    with tempfile.TemporaryDirectory(prefix="plfbs_refcpu_") as wd:
        cases.write_polymesh(os.path.join(wd, "polyMesh"), pm)
        t_setup = _run_ref_cpu(wd, pm, c, nodes, 0)
        t_run = _run_ref_cpu(wd, pm, c, nodes, sample_steps)
    per_step = max(t_run - t_setup, 1e-9) / sample_steps
    return pm.n_cells / per_step / 1e6, (
        "%d time step(s) of the reference CPU Solver on the same %dx%dx%d mesh and boundary "
        "conditions (the CPU Solver has no IBM), timed from its \"Running Solver\" line with "
        "the solver's setup subtracted via a 0-step run (%.1f s setup, %.1f s per step), "
        "serial" % (sample_steps, NX, NY, NZ, t_setup, per_step))


REF_GPU_BIN = os.path.join(REPO, "oracle", "_ref", "plfbs_ref_gpu")


def reference_gpu_throughput(pm, c, nodes, steps=2001, every=100, limit=600):
    """Mcell-updates/s of the reference's own CUDA path (oracle/_ref/plfbs_ref_gpu:
    Solver_gpu.cu and its kernels built for sm_100a) on the same case: it prints
    a progress line every `every` steps (Solver_gpu.cu:844-853), and the median
    time between their arrivals, over `every`, is its time per step with its
    setup and the occasional decade output left out."""
    import copy
    if not os.path.exists(REF_GPU_BIN):
        return None, "oracle/_ref/plfbs_ref_gpu not built"
    c = copy.copy(c)
    stamps, rc = [], None
    with tempfile.TemporaryDirectory(prefix="plfbs_refgpu_") as wd:
        cases.write_polymesh(os.path.join(wd, "polyMesh"), pm)
        node_file = os.path.join(wd, "nodes.txt")
        cases.write_spring_network(node_file, nodes)
        c.steps, c.gpu_solver, c.output_step = steps, 1, every
        c.output_dir = os.path.join(wd, "out") + "/"
        c.obj_nodes_file, c.obj_num_nodes = node_file, len(nodes)
        c.mesh_dir = os.path.join(wd, "polyMesh")
        xml = os.path.join(wd, "case.xml")
        cases.write_xml(xml, c)
        p = subprocess.Popen([REF_GPU_BIN, xml], cwd=wd, stdout=subprocess.PIPE,
                             stderr=subprocess.DEVNULL, text=True)
        timer = threading.Timer(limit, p.kill)  # this process only
        timer.start()
        try:
            for line in p.stdout:
                if line.startswith("time t="):
                    stamps.append(time.perf_counter())
            rc = p.wait()
        finally:
            timer.cancel()
    if rc != 0 or len(stamps) < 3:
        return None, "the reference CUDA path exited with %s after %d progress lines" % (
            rc, len(stamps))
    gaps = sorted(b - a for a, b in zip(stamps, stamps[1:]))
    per_step = gaps[len(gaps) // 2] / every
    return pm.n_cells / per_step / 1e6, (
        "the reference's Solver_gpu.cu path built for sm_100a on the same case (IBM included), "
        "%d steps, median of %d intervals of %d steps between its progress lines (setup and "
        "decade outputs left out), %.3f ms per step" % (steps, len(gaps), every, 1e3 * per_step))


def _mem_available():
    """MemAvailable of the host in bytes (None if unknown)."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return None


def reference_cpu_aggregate(pm, c, nodes, steps=11, every=2):
    """Mcell-updates/s of the reference CPU Solver on all the host threads it
    can use: the Solver is serial, so P independent instances run at once, P
    the threads available to this process, bounded so that P times one
    instance's peak memory stays within half of MemAvailable and P times its
    files (about 100 MB of text output) within half of the free space of the
    temporary directory. Each instance
    runs `steps` steps printing a progress line every `every` steps
    (Solver.cpp:501-508); the Solver writes its text output after a progress
    line only while its residual crosses a new decade (the first few lines),
    so an instance's step time is the shorter of its last two intervals over
    `every`. The aggregate is the sum of the instances' rates. Returns
    (value, cores, sample)."""
    import copy
    import resource
    from concurrent.futures import ThreadPoolExecutor
    v1, sample1 = reference_cpu_throughput(pm, copy.copy(c), nodes, sample_steps=1)
    if v1 is None:
        return None, 0, sample1
    threads = len(os.sched_getaffinity(0))
    rss = resource.getrusage(resource.RUSAGE_CHILDREN).ru_maxrss * 1024  # one instance's peak
    avail = _mem_available()
    P = threads if not avail or rss <= 0 else max(1, min(threads, int(0.5 * avail // rss)))
    import shutil
    P = max(1, min(P, int(0.5 * shutil.disk_usage(tempfile.gettempdir()).free // (128 << 20))))
    if P == 1:
        return v1, 1, sample1
    with tempfile.TemporaryDirectory(prefix="plfbs_refcpu_") as wd:
        mesh_dir = os.path.join(wd, "polyMesh")
        cases.write_polymesh(mesh_dir, pm)

        def instance(i):
            d = os.path.join(wd, "i%d" % i)
            os.makedirs(d)
            ci = copy.copy(c)
            ci.output_step = every
            stamps = []
            _run_ref_cpu(d, pm, ci, nodes, steps, mesh_dir, progress=stamps)
            gaps = [b - a for a, b in zip(stamps, stamps[1:])]
            return min(gaps[-2:]) / every if len(gaps) >= 2 else None

        try:
            with ThreadPoolExecutor(max_workers=P) as ex:
                per_step = list(ex.map(instance, range(P)))
        except Exception as e:  # the single-instance figure stands
            return v1, 1, sample1 + "; %d concurrent instances failed (%s)" % (P, e)
    if any(t is None or t <= 0 for t in per_step):
        return v1, 1, sample1 + "; %d concurrent instances gave no step time" % P
    value = sum(pm.n_cells / t / 1e6 for t in per_step)
    return value, P, (
        "%d concurrent instances of the serial reference CPU Solver (the host threads "
        "available, within half of MemAvailable at %.2f GB per instance and half of the free "
        "temporary disk space), each %d time steps of "
        "the same %d-cell mesh timed between its progress lines every %d steps past its "
        "decade outputs (%.3g-%.3g s per step); sum of their rates. One instance alone: "
        "%.3f Mcell-updates/s" % (P, rss / 1e9, steps, pm.n_cells, every, min(per_step),
                                  max(per_step), v1))


def reduce_max(x, dist=None, device="cuda"):
    """Max of a float over the ranks of a process group (identity without one)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, cells, steps, max_ms):
    """Whole-job Mcell-updates/s of `world` independent replicas, each updating
    `cells` cells for `steps` steps, timed by the slowest rank."""
    return world * cells * steps / (max_ms / 1e3) / 1e6


# ---------------------------------------------------------------------------
# time to a residual: FP64 vs the FP32 deviation form from the same cold start
# ---------------------------------------------------------------------------

TTR_WORKLOAD = "sphere_channel_64x32x32_D8_re100"


def build_ttr_case(nx=64, ny=32, nz=32, D=8.0, re=100.0):
    """The learned-warm-start geometry (64 x 32 x 32 channel, sphere D = 8 at
    (16, 16, 16), Fibonacci nodes at the node density of the headline case)."""
    pm = cases.uniform_box(nx, ny, nz, patch_types=["inlet", "outlet", "side", "side", "side",
                                                    "side"])
    c = cases.Case(mesh_dir="", X=nx, Y=ny, Z=nz, dt=DT, mach=U, reynolds=re, ref_length=D,
                   tolerance=0.0,
                   bcs=[cases.BC("inlet", 1, 1, 0, 0, "dirichlet", "neumann"),
                        cases.BC("outlet", 1, 0, 0, 0, "neumann", "dirichlet"),
                        cases.BC("side", 1, 0, 0, 0, "neumann", "neumann")])
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    n_nodes = int(round(4 * np.pi * (D / 2) ** 2 / (4 * np.pi * (DIAM / 2) ** 2 / NNODES)))
    nodes = cases.fibonacci_sphere(n_nodes, D / 2, (2 * D, ny / 2, nz / 2))
    state0 = np.zeros((ma.total_cells, 4))
    state0[:, 0] = U
    state0[:, 3] = 1.0
    ibm = dict(node_ref=nodes, stiffness=STIFFNESS, radius=D / 2, depth=D,
               object_nodes=len(nodes))
    return c, ma, state0, ibm, np.pi * D * D / 4


def time_to_residual(args):
    from plfbs import capi

    c, ma, state0, ibm, area = build_ttr_case()
    rt, vt, val = cases.bc_arrays(ma, c)
    out, states = {}, {}
    for name, prec in (("fp64", capi.FP64), ("fp32", capi.FP32_DEVIATION)):
        cfg = solver_cfg(c, prec)
        cfg["tolerance"] = args.time_to_residual
        s = capi.Solver(ma, rt, vt, val, cfg, ibm=ibm)
        s.set_state(state0)
        t0 = time.perf_counter()
        st, hist = s.run(args.max_steps, history=False)
        wall = time.perf_counter() - t0
        cd, cl = s.body_force(area)
        states[name] = s.get_state()
        s.close()
        out[name] = {"converged": bool(st["converged"]), "steps": st["steps_done"],
                     "device_s": st["kernel_ms"] / 1e3, "wall_s": wall,
                     "final_max_error": st["max_error"], "cd": cd, "cl": cl}
    # FP32 from the trained network's prediction (plfbs/data/warmstart_params.npz);
    # the same channel, sphere and Re (a member of the network's training family)
    from plfbs import warmstart
    if os.path.exists(warmstart.PARAMS):
        centre = (2 * 8.0, 16.0, 16.0)
        t0 = time.perf_counter()
        ws = warmstart.WarmStarter()
        t1 = time.perf_counter()
        start = ws.start(100.0, centre)
        infer = time.perf_counter() - t1
        rec, q = ws.ch.solve(100.0, centre, capi.FP32_DEVIATION, args.time_to_residual,
                             args.max_steps, start=start)
        ws.close()
        rec.update(nn_inference_s=infer, nn_setup_s=t1 - t0,
                   wall_s_with_inference=rec["wall_s"] + infer)
        out["fp32_nn"] = rec
        states["fp32_nn"] = q
    a, b = states["fp64"], states["fp32"]
    err = {k: float(np.linalg.norm(b[:, i] - a[:, i]) / np.linalg.norm(a[:, i]))
           for i, k in enumerate(("u", "v", "w"))}
    err["rho-rho0"] = float(np.linalg.norm(b[:, 3] - a[:, 3]) / np.linalg.norm(a[:, 3] - 1.0))
    line = {"metric": "time-to-residual", "tolerance": args.time_to_residual,
            "unit": "s", "higher_is_better": False, "data": "synthetic",
            "config": {"workload": TTR_WORKLOAD, "cells": ma.n_cells, "faces": ma.n_faces,
                       "nodes": len(ibm["node_ref"]), "start": "uniform flow (cold)"},
            "fp64": out["fp64"], "fp32": out["fp32"], "fp32_nn": out.get("fp32_nn"),
            "speedup_fp32_over_fp64": out["fp64"]["wall_s"] / out["fp32"]["wall_s"],
            "speedup_fp32_nn_over_fp64": (out["fp64"]["wall_s"] /
                                          out["fp32_nn"]["wall_s_with_inference"]
                                          if "fp32_nn" in out else None),
            "fp32_vs_fp64_rel_l2": err,
            "cd_rel_diff": abs(out["fp32"]["cd"] - out["fp64"]["cd"]) / abs(out["fp64"]["cd"])}
    print(json.dumps(line))
    return 0


def compare_precisions(args):
    """FP32 deviation form against the FP64 path on the other configurations:
    `tets` = 64^3 unit hexes with interior nodes jittered (seeded), each split
    into 6 tetrahedra (1,572,864 cells), Taylor-Green initial field (U 0.05),
    Re 400 on L = 64, Dirichlet u = 0 walls, 500 steps of dt 0.05, exact-inverse
    least squares (the reference's determinant is unstable on tets). Jitter
    +-0.1 of the spacing: at +-0.2 the scheme diverges near t = 4.5 whatever
    Re, U or dt (a mesh-quality instability), at +-0.1 and below it does not;
    `scale` = 256 x 128 x 128 channel, sphere D 32 at (64, 64, 64) with 12,869
    nodes, Re 200, 2000 steps. One JSON line: throughput, the flux kernel's
    fraction of the measured HBM bandwidth, per-field relative L2 of FP32
    against FP64, and (scale) Cd of both."""
    from plfbs import capi
    if args.compare == "tets":
        n, u0, re, steps = 64, 0.05, 400.0, 500
        pm = cases.jittered_tet_box(n, jitter=args.jitter, seed=11, patch_types=["wall"] * 6)
        c = cases.Case(mesh_dir="", X=n, Y=n, Z=n, dt=args.compare_dt or 0.05, mach=u0,
                       reynolds=re, ref_length=n,
                       bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann")])
        ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
        x = np.asarray(ma.cell_centroid).reshape(-1, 3) * (2 * np.pi / n)
        state0 = np.zeros((ma.total_cells, 4))
        state0[:, 0] = u0 * np.sin(x[:, 0]) * np.cos(x[:, 1]) * np.cos(x[:, 2])
        state0[:, 1] = -u0 * np.cos(x[:, 0]) * np.sin(x[:, 1]) * np.cos(x[:, 2])
        state0[:, 3] = 1.0
        ibm, area, mode = None, None, capi.GRAD_EXACT_INVERSE
        name = "tgv_tets_64cubed_jitter%g_re400" % args.jitter
    else:
        nx, ny, nz, d, re, steps = 256, 128, 128, 32.0, 200.0, 2000
        pm = cases.uniform_box(nx, ny, nz, patch_types=["inlet", "outlet", "side", "side",
                                                        "side", "side"])
        c = cases.Case(mesh_dir="", X=nx, Y=ny, Z=nz, dt=DT, mach=U, reynolds=re,
                       ref_length=d, tolerance=0.0,
                       bcs=[cases.BC("inlet", 1, 1, 0, 0, "dirichlet", "neumann"),
                            cases.BC("outlet", 1, 0, 0, 0, "neumann", "dirichlet"),
                            cases.BC("side", 1, 0, 0, 0, "neumann", "neumann")])
        ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
        nodes = cases.fibonacci_sphere(12869, d / 2, (64.0, 64.0, 64.0))
        ibm = dict(node_ref=nodes, stiffness=STIFFNESS, radius=d / 2, depth=d,
                   object_nodes=len(nodes))
        state0 = np.zeros((ma.total_cells, 4))
        state0[:, 0] = U
        state0[:, 3] = 1.0
        area, mode = np.pi * d * d / 4, 0
        name = "sphere_channel_256x128x128_ibm12869_re200"
    rt, vt, val = cases.bc_arrays(ma, c)
    peak, peak_kind = load_peaks()
    out, states = {}, {}
    for prec_name, prec in (("fp64", capi.FP64), ("fp32", capi.FP32_DEVIATION)):
        cfg = solver_cfg(c, prec)
        cfg["gradient_mode"] = mode
        s = capi.Solver(ma, rt, vt, val, cfg, ibm=ibm)
        s.set_state(state0)
        st, _ = s.run(steps, history=False)
        if st["rc"] != 0 or st["steps_done"] != steps:
            print(json.dumps({"metric": "fp32-vs-fp64", "config": {"workload": name},
                              "failed": "%s stopped after %d steps (status %d)"
                              % (prec_name, st["steps_done"], st["rc"])}))
            return 1
        r = {"steps": int(st["steps_done"]), "ms_per_step": st["kernel_ms"] / steps,
             "mcell_updates_per_s": ma.n_cells * steps / st["kernel_ms"] / 1e3}
        prof = s.profile_steps(10)
        flux_ms = prof["flux"] / 40
        alg = algorithmic_bytes(ma.n_cells, ma.n_faces, ma.n_bc, fp32=prec_name == "fp32")
        r["flux_ms"] = flux_ms
        r["flux_hbm_frac"] = alg["flux"] / (flux_ms / 1e3) / 1e9 / peak
        s.set_state(state0)
        s.run(steps, history=False)  # the same state after exactly `steps` steps
        if area:
            r["cd"], r["cl"] = s.body_force(area)
        states[prec_name] = s.get_state()
        s.close()
        out[prec_name] = r
    a, b = states["fp64"][: ma.n_cells], states["fp32"][: ma.n_cells]
    err = {k: float(np.linalg.norm(b[:, i] - a[:, i]) / np.linalg.norm(a[:, i]))
           for i, k in enumerate(("u", "v", "w"))}
    err["rho-rho0"] = float(np.linalg.norm(b[:, 3] - a[:, 3]) / np.linalg.norm(a[:, 3] - 1.0))
    line = {"metric": "fp32-vs-fp64", "config": {"workload": name, "cells": ma.n_cells,
                                                 "faces": ma.n_faces, "steps": steps},
            "peak_gbs": peak, "peak_kind": peak_kind, "fp64": out["fp64"], "fp32": out["fp32"],
            "fp32_vs_fp64_rel_l2": err}
    if area:
        line["cd_rel_diff"] = abs(out["fp32"]["cd"] - out["fp64"]["cd"]) / abs(out["fp64"]["cd"])
    print(json.dumps(line))
    return 0


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    pm, c, ma, nodes, _ = build_case()
    value, cores, sample = reference_cpu_aggregate(pm, c, nodes)
    cfg = {"workload": WORKLOAD, "cells": ma.n_cells, "faces": ma.n_faces,
           "nodes": NNODES, "re": RE, "dt": DT,
           "parallelism": "replicas" if world > 1 else "single"}
    if value is None:
        print(json.dumps({"impl": "reference", "unavailable": sample}))
        return 0
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
            "n_gpus": world, "steps": 1, "warmup": 0, "requested_steps": args.steps,
            "ms_per_step": ma.n_cells / value / 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def log(msg):
    print("[bench] %s" % msg, file=sys.stderr, flush=True)


def main():
    faulthandler.enable()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--renumber", type=int, default=0, choices=[0, 1, 2],
                    help="cell order: 0 the mesh's (blockMesh), 1 RCM on the host, 2 on the device")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own CUDA path on the same case")
    ap.add_argument("--profile-steps", type=int, default=20)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="fp32: the FP32 deviation form (the headline line is fp64)")
    ap.add_argument("--time-to-residual", type=float, default=None,
                    help="instead of throughput: steps and time to max_error < this value, "
                         "FP64 vs FP32 from a cold start")
    ap.add_argument("--max-steps", type=int, default=100000)
    ap.add_argument("--compare", choices=["tets", "scale"], default=None,
                    help="instead of throughput: FP32 vs FP64 on another configuration")
    ap.add_argument("--compare-dt", type=float, default=None, help="RK dt of the tets case")
    ap.add_argument("--jitter", type=float, default=0.1, help="node jitter of the tets case")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.time_to_residual is not None:
        return time_to_residual(args) if rank == 0 else 0
    if args.compare is not None:
        return compare_precisions(args) if rank == 0 else 0

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from plfbs import capi

    pm, c, ma, nodes, state0 = build_case()
    rt, vt, val = cases.bc_arrays(ma, c)
    log("case built: %d cells, %d faces" % (ma.n_cells, ma.n_faces))
    prec = capi.FP32_DEVIATION if args.precision == "fp32" else capi.FP64
    solver = capi.Solver(ma, rt, vt, val, solver_cfg(c, prec, args.renumber), ibm=ibm_cfg(nodes),
                         device=local_rank)

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_max(x, dist, "cuda")

    log("solver created")
    # warm-up
    solver.set_state(state0)
    st, _ = solver.run(args.warmup, history=False)
    if st["rc"] != 0:
        raise RuntimeError("warm-up diverged")
    barrier()
    with ClockSampler(local_rank) as clk:
        st, hist = solver.run(args.steps, history=True)
    barrier()
    if st["rc"] != 0 or st["steps_run"] != args.steps:
        raise RuntimeError("timed run stopped early: %r" % st)
    ms = max_over_ranks(st["kernel_ms"])
    value = replica_throughput(world, ma.n_cells, args.steps, ms)

    log("timed run: %.3f ms for %d steps" % (ms, args.steps))
    # per-kernel device times (CUDA events between launches on the solver's stream)
    prof = solver.profile_steps(args.profile_steps)
    log("profile: %r" % prof)
    per_launch = {"ibm": prof["ibm"] / args.profile_steps,
                  "gradient": prof["gradient"] / (4 * args.profile_steps),
                  "flux": prof["flux"] / (4 * args.profile_steps),
                  "update": prof["update"] / (4 * args.profile_steps)}
    total = sum(prof.values())
    workload = WORKLOAD if args.precision == "fp64" else WORKLOAD.replace("fp64", "fp32dev")
    if args.renumber:  # another cell order: the committed traffic figures do not apply
        workload += "_rcm"
    alg = algorithmic_bytes(ma.n_cells, ma.n_faces, ma.n_bc, fp32=args.precision == "fp32")
    peak, peak_kind = load_peaks()
    kern = {}
    for k in ("gradient", "flux", "update"):
        gbs = alg[k] / (per_launch[k] / 1e3) / 1e9
        kern[k] = {"ms_per_launch": per_launch[k], "share": prof[k] / total,
                   "algorithmic_bytes": alg[k], "achieved_gbs": gbs, "frac": gbs / peak}
    kern["ibm"] = {"ms_per_launch": per_launch["ibm"], "share": prof["ibm"] / total}
    dom = max(("gradient", "flux", "update"), key=lambda k: prof[k])
    roof = {"kernel": dom, "bound": "hbm", "achieved": kern[dom]["achieved_gbs"], "peak": peak,
            "unit": "GB/s", "frac": kern[dom]["frac"], "peak_kind": peak_kind,
            "traffic": load_traffic(dom, workload)}

    # end to end through the C ABI from host buffers; the median of E2E_REPS
    # repetitions (host-side timings on a shared machine vary from run to run)
    e2e = None
    if not args.no_e2e:
        barrier()
        solver.close()
        reps = []
        for _ in range(E2E_REPS):
            barrier()
            t0 = time.perf_counter()
            s2 = capi.Solver(ma, rt, vt, val, solver_cfg(c, prec, args.renumber),
                             ibm=ibm_cfg(nodes),
                             device=local_rank)
            t1 = time.perf_counter()
            s2.set_state(state0)
            t2 = time.perf_counter()
            st2, hist2 = s2.run(args.steps, history=True)
            t3 = time.perf_counter()
            out = s2.get_state()
            t4 = time.perf_counter()
            s2.close()
            t5 = time.perf_counter()
            reps.append((max_over_ranks(t5 - t0),
                         {"create_s": t1 - t0, "set_state_s": t2 - t1, "run_s": t3 - t2,
                          "get_state_s": t4 - t3, "destroy_s": t5 - t4}))
            assert np.isfinite(out).all() and st2["steps_run"] == args.steps
        reps.sort(key=lambda r: r[0])
        wall, phases = reps[len(reps) // 2]
        T = ma.total_cells
        mesh_bytes = (ma.n_faces * (4 + 4 + 8 + 24 + 24 + 8) + T * (8 + 24) +
                      (ma.n_cells + 1 + 2 * len(ma.stencil_cells)) * 4 + ma.n_bc * (4 + 4 + 32) +
                      len(nodes) * 48)
        h2d = mesh_bytes + T * 32
        d2h = T * 32 + 48 * args.steps
        e2e = {"value": replica_throughput(world, ma.n_cells, args.steps, wall * 1e3),
               "unit": METRIC,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "wall_s": wall, "includes": "create+set_state+run+history+get_state+destroy",
               "repetitions": E2E_REPS, "of": "median", "walls_s": [r[0] for r in reps],
               "phases": phases}
    else:
        solver.close()

    log("e2e: %r" % e2e)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sample = reference_cpu_throughput(pm, c, nodes, sample_steps=1)
        if v is not None:
            cpu = {"value": v, "unit": METRIC, "cores": 1, "kind": "reference", "sample": sample}
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu and args.precision == "fp64":
        v, sample = reference_gpu_throughput(pm, c, nodes)
        ref_gpu = {"value": v, "unit": METRIC, "sample": sample}
        log("reference GPU: %r" % ref_gpu)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32", "data": "synthetic",
                "config": {"workload": workload, "cells": ma.n_cells, "faces": ma.n_faces,
                           "nodes": NNODES, "re": RE, "dt": DT,
                           "parallelism": "replicas" if world > 1 else "single",
                           "renumber": args.renumber,
                           "l2": "working set > L2 (no flush)"},
                "per_rk_stage": {"value": 4 * value, "unit": "Mcell-stage-updates/s"},
                "roofline": roof, "kernels": kern, "cpu_baseline": cpu,
                "reference_gpu": ref_gpu, "e2e": e2e,
                "gpu_launches": KERNELS_PER_STEP * args.steps, "clocks": clk.summary(),
                "final_max_error": float(hist[-1, 1]) if len(hist) else None}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
