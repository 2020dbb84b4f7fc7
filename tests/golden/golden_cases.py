"""Definitions of the small seeded cases behind the committed golden fixtures.

Shared by make_golden.py (which runs the reference on them) and the tests
(which rebuild the same inputs and compare against the fixtures). Each case
exercises a different part of the reference's GPU path:

  cavity    6x5x4 lid-driven cavity, Dirichlet walls + moving lid, LS weights
  channel   10x6x6 channel: parabolic inlet (vel type 9), pressure outlet,
            no-slip and Neumann walls, a body force, an IBM sphere of 30
            Fibonacci nodes plus two nodes near x = 0 whose structured index
            wraps across rows (the reference checks only the linear index)
  graded    6x6x5 geometrically graded hexes, hybrid LS/Green-Gauss weights,
            gamma = 1.3, streaming dt capped by fneq_min, offset origin
  converge  the cavity with a loose tolerance: stops after its first step

and of the reference CPU Solver (Solver.cpp), no IBM, from a seeded field:

  cpu_cavity   6x5x4 cavity, Dirichlet walls and lid, Neumann density
  cpu_channel  10x6x6 channel, gamma = 1.2, a body force: velocity "inlet" (6),
               Dirichlet-density outlet, "symmetry-x" (8) sides in y, no-slip
               walls in z with density "wall" (7)
  cpu_tets     4x4x4 hexes with jittered nodes split into 384 tetrahedra, walls
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "3d-plfbs-gpu_b200"))

from plfbs import cases  # noqa: E402

NAMES = ("cavity", "channel", "graded", "converge")
CPU_NAMES = ("cpu_cavity", "cpu_channel", "cpu_tets")


def _random_state(ma, seed, amp=0.02):
    rng = np.random.Generator(np.random.PCG64(seed))
    T = ma.total_cells
    x = ma.cell_centroid
    s = np.zeros((T, 4))
    s[:, 0] = amp * np.sin(0.7 * x[:, 0] + 0.3 * x[:, 2]) + 0.5 * amp * rng.standard_normal(T)
    s[:, 1] = amp * np.cos(0.5 * x[:, 1]) + 0.5 * amp * rng.standard_normal(T)
    s[:, 2] = 0.5 * amp * np.sin(x[:, 2] + x[:, 0]) + 0.5 * amp * rng.standard_normal(T)
    s[:, 3] = 1.0 + 0.5 * amp * rng.standard_normal(T)
    return s


def build(name):
    """Returns dict(pm, case, nodes, state0, ma) for a golden case."""
    if name in ("cavity", "converge"):
        pm = cases.uniform_box(6, 5, 4, patch_types=["wall", "wall", "wall", "lid", "wall", "wall"])
        c = cases.Case(mesh_dir="", X=6, Y=5, Z=4, steps=3, dt=0.1, mach=0.1, reynolds=100,
                       ref_length=6, obj_centre=(3.0, 2.5, 2.0),
                       bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann"),
                            cases.BC("lid", 1, 1, 0, 0, "dirichlet", "neumann")])
        if name == "converge":
            c.tolerance = 1.0
            c.steps = 5
        nodes = np.array([[3.0, 2.5, 2.0]])
        seed = 11
    elif name == "channel":
        pm = cases.uniform_box(10, 6, 6, patch_types=["inlet", "outlet", "wall", "wall",
                                                      "side", "side"])
        c = cases.Case(mesh_dir="", X=10, Y=6, Z=6, steps=3, dt=0.2, mach=0.05, reynolds=20,
                       ref_length=3, pressure_gradient=1e-4,
                       bcs=[cases.BC("inlet", 1, 1, 0, 0, "parabolic", "neumann"),
                            cases.BC("outlet", 1, 0, 0, 0, "neumann", "dirichlet"),
                            cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann"),
                            cases.BC("side", 1, 0, 0, 0, "neumann", "neumann")])
        sphere = cases.fibonacci_sphere(30, 1.5, (4.0, 3.0, 3.0))
        edge = np.array([[0.2, 2.4, 3.3], [0.6, 4.5, 1.2]])
        nodes = np.concatenate([sphere, edge])
        c.obj_radius, c.obj_depth, c.obj_stiffness = 1.5, 3.0, 0.3
        c.obj_centre = (4.0, 3.0, 3.0)
        seed = 12
    elif name == "graded":
        g = lambda n, r: np.concatenate([[0.0], np.cumsum(r ** np.arange(n))])  # noqa: E731
        xs, ys, zs = 0.5 + g(6, 1.15), -1.0 + g(6, 0.9), 2.0 + g(5, 1.25)
        pm = cases.hex_box(xs, ys, zs, patch_types=["in", "out", "wall", "wall", "wall", "top"])
        c = cases.Case(mesh_dir="", X=float(xs[-1] - xs[0]), Y=float(ys[-1] - ys[0]),
                       Z=float(zs[-1] - zs[0]), origin=(0.5, -1.0, 2.0), steps=3, dt=0.05,
                       mach=0.1, reynolds=100, ref_length=6, gamma=1.3,
                       gradient_calc="hybrid", fneq_min=0.036,
                       bcs=[cases.BC("in", 1.01, 0.5, 0.1, 0, "dirichlet", "neumann"),
                            cases.BC("out", 0.99, 0, 0, 0, "neumann", "dirichlet"),
                            cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann"),
                            cases.BC("top", 1, 0.3, 0, 0.2, "dirichlet", "dirichlet")])
        nodes = np.array([[2.0, 1.0, 3.0]])
        c.obj_centre = (2.0, 1.0, 3.0)
        seed = 13
    else:
        raise KeyError(name)
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    state0 = _random_state(ma, seed)
    return dict(pm=pm, case=c, nodes=nodes, state0=state0, ma=ma)


def build_cavity32(cpu_solver=False, steps=2000):
    """The plain-method lid-driven cavity at full size: a 32^3 uniform hex
    unit cube (lattice units, dx = 1), Re 100 on L = 32, lid velocity 0.1
    (Dirichlet velocity, Neumann density on every wall), dt 0.18, from rest
    (u = 0, rho = 1), `steps` RK4 steps. Returns dict(pm, case, nodes,
    state0, ma)."""
    n = 32
    pm = cases.uniform_box(n, n, n, patch_types=["wall", "wall", "wall", "lid", "wall", "wall"])
    c = cases.Case(mesh_dir="", X=n, Y=n, Z=n, steps=steps, dt=0.18, mach=0.1, reynolds=100,
                   ref_length=n, tolerance=0.0, gpu_solver=0 if cpu_solver else 1,
                   obj_centre=(16.0, 16.0, 16.0),
                   bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann"),
                        cases.BC("lid", 1, 1, 0, 0, "dirichlet", "neumann")])
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    s0 = np.zeros((ma.total_cells, 4))
    s0[:, 3] = 1.0
    nodes = np.zeros((0, 3)) if cpu_solver else np.array([[16.0, 16.0, 16.0]])
    return dict(pm=pm, case=c, nodes=nodes, state0=s0, ma=ma)


def build_tgv_tets(n=12, jitter=0.2, gradient_calc="GG", steps=100, seed=11):
    """The unstructured stress case at small size: n^3 hexes with interior
    nodes jittered uniformly by +-jitter of the spacing (seeded), each split
    into 6 tetrahedra, no-slip walls (Dirichlet velocity, Neumann density), a
    Taylor-Green field of amplitude 0.05 at rest density, Re 400 on L = n,
    dt 0.05. Green-Gauss gradients by default: their 2 V I matrix inverts
    exactly under the reference's cofactor formula, so the reference itself
    runs tetrahedra with a sound gradient (its least-squares inverse does not,
    gradients.cpp:282-284). Returns dict(pm, case, nodes, state0, ma)."""
    u0 = 0.05
    pm = cases.jittered_tet_box(n, jitter=jitter, seed=seed, patch_types=["wall"] * 6)
    c = cases.Case(mesh_dir="", X=n, Y=n, Z=n, dt=0.05, mach=u0, reynolds=400.0, ref_length=n,
                   tolerance=0.0, steps=steps, gpu_solver=0, gradient_calc=gradient_calc,
                   bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann")])
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    x = np.asarray(ma.cell_centroid).reshape(-1, 3) * (2 * np.pi / n)
    s0 = np.zeros((ma.total_cells, 4))
    s0[:, 0] = u0 * np.sin(x[:, 0]) * np.cos(x[:, 1]) * np.cos(x[:, 2])
    s0[:, 1] = -u0 * np.cos(x[:, 0]) * np.sin(x[:, 1]) * np.cos(x[:, 2])
    s0[:, 3] = 1.0
    return dict(pm=pm, case=c, nodes=np.zeros((0, 3)), state0=s0, ma=ma)


def failure_step(lines):
    """The step at which the reference CPU Solver stopped on a diverged field
    ("rho failure" / "nan failure" followed by the step, Solver.cpp:448-493),
    or None."""
    for k, line in enumerate(lines):
        if line.strip() in ("rho failure", "nan failure"):
            return int(lines[k + 1])
    return None


def oracle_cfg(d):
    """The scalar configuration the solver sees for a golden case."""
    c = d["case"]
    nodes = d["nodes"]
    return dict(visc=c.visc, gamma=c.gamma, dt=c.dt, domain_dt=c.streaming_dt,
                pressure_gradient=c.pressure_gradient, channel_height=c.Y,
                max_velocity=c.mach, ref_rho=c.average_rho, tolerance=c.tolerance,
                origin=c.origin, lengths=(c.X, c.Y, c.Z),
                gradient_mode={"LS": 0, "hybrid": 1}.get(c.gradient_calc, 2),
                node_ref=nodes, node_x=nodes, stiffness=c.obj_stiffness, radius=c.obj_radius,
                depth=c.obj_depth, object_nodes=nodes.shape[0])


def build_cpu(name):
    """Returns dict(pm, case, nodes, state0, ma) for a CPU-Solver case."""
    if name == "cpu_cavity":
        pm = cases.uniform_box(6, 5, 4, patch_types=["wall", "wall", "wall", "lid", "wall", "wall"])
        c = cases.Case(mesh_dir="", X=6, Y=5, Z=4, dt=0.1, mach=0.1, reynolds=100.0,
                       ref_length=4.0, tolerance=0.0, steps=25, gpu_solver=0,
                       bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann"),
                            cases.BC("lid", 1, 1, 0, 0, "dirichlet", "neumann")])
        seed = 21
    elif name == "cpu_channel":
        pm = cases.uniform_box(10, 6, 6, patch_types=["inlet", "outlet", "slip", "slip", "wall",
                                                      "wall"])
        c = cases.Case(mesh_dir="", X=10, Y=6, Z=6, dt=0.1, mach=0.05, reynolds=50.0,
                       ref_length=6.0, tolerance=0.0, steps=20, gpu_solver=0, gamma=1.2,
                       pressure_gradient=2e-5,
                       bcs=[cases.BC("inlet", 1, 1, 0, 0, "inlet", "neumann"),
                            cases.BC("outlet", 1, 0, 0, 0, "neumann", "dirichlet"),
                            cases.BC("slip", 1, 0, 0, 0, "symmetry-x", "neumann"),
                            cases.BC("wall", 1, 0, 0, 0, "dirichlet", "wall")])
        seed = 22
    elif name == "cpu_tets":
        pm = cases.jittered_tet_box(4, jitter=0.1, seed=23,
                                    patch_types=["wall", "wall", "wall", "lid", "wall", "wall"])
        c = cases.Case(mesh_dir="", X=4, Y=4, Z=4, dt=0.05, mach=0.1, reynolds=100.0,
                       ref_length=4.0, tolerance=0.0, steps=10, gpu_solver=0,
                       bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann"),
                            cases.BC("lid", 1, 1, 0, 0, "dirichlet", "neumann")])
        seed = 24
    else:
        raise KeyError(name)
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    return dict(pm=pm, case=c, nodes=np.zeros((0, 3)), state0=_random_state(ma, seed), ma=ma)
