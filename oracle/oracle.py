"""ORACLE — test infrastructure only. ctypes front end of plfbs_oracle.c, the
plain-C FP64 restatement of the reference's GPU time step.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker. ``build()`` compiles the C file with gcc
into oracle/lib/liboracle.so (no GPU, no CUDA).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "plfbs_oracle.c")
LIB = os.path.join(HERE, "lib", "liboracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Problem(C.Structure):
    _fields_ = [("n_cells", C.c_int), ("n_faces", C.c_int), ("n_internal", C.c_int),
                ("owner", _ip), ("neighbour", _ip), ("face_area", _dp), ("face_normal", _dp),
                ("face_centroid", _dp), ("streaming_dt", _dp), ("cell_volume", _dp),
                ("cell_centroid", _dp), ("st_off", _ip), ("st_cells", _ip), ("st_faces", _ip),
                ("bc_rho_type", _ip), ("bc_vel_type", _ip), ("bc_value", _dp),
                ("lhs_inv", _dp), ("rhs", _dp), ("visc", C.c_double), ("gamma", C.c_double),
                ("dt", C.c_double), ("domain_dt", C.c_double),
                ("pressure_gradient", C.c_double), ("channel_height", C.c_double),
                ("max_velocity", C.c_double), ("ref_rho", C.c_double),
                ("tolerance", C.c_double), ("origin", C.c_double * 3),
                ("lengths", C.c_double * 3), ("n_nodes", C.c_int), ("object_nodes", C.c_int),
                ("node_ref", _dp), ("stiffness", C.c_double), ("radius", C.c_double),
                ("depth", C.c_double), ("flavour", C.c_int)]


class _State(C.Structure):
    _fields_ = [("state", _dp), ("t0", _dp), ("t1", _dp), ("node_x", _dp), ("node_x0", _dp),
                ("node_vel", _dp), ("node_force", _dp), ("force", _dp), ("grad", _dp),
                ("face_flux", _dp), ("residual", _dp), ("history", _dp), ("stage", C.c_int)]


def build(force=False):
    """Compile liboracle.so with gcc (-O2, no FMA contraction on x86-64)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    tmp = LIB + ".tmp%d" % os.getpid()
    subprocess.run(["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-ffp-contract=off", SRC,
                    "-o", tmp, "-lm"], check=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.oracle_ls_weights.restype = C.c_int
        _lib.oracle_run.restype = C.c_int
        _lib.oracle_run.argtypes = [C.POINTER(_Problem), C.POINTER(_State), C.c_int, C.c_int]
        _lib.oracle_init_t1.argtypes = [C.POINTER(_Problem), C.POINTER(_State)]
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def ls_weights(ma, mode):
    """(lhs_inv [C,3,3], rhs [nnz,3]) as gradients::pre_fill_LHS_and_RHS_matrix
    computes them; mode 0 = LS, 1 = hybrid, 2 = Green-Gauss."""
    nnz = int(ma.stencil_offsets[-1])
    lhs = np.zeros((ma.n_cells, 3, 3))
    rhs = np.zeros((nnz, 3))
    arrs = [np.ascontiguousarray(x) for x in (
        ma.stencil_offsets, ma.stencil_cells, ma.stencil_faces, ma.owner, ma.face_area,
        ma.face_normal, ma.face_centroid, ma.cell_volume, ma.cell_centroid)]
    lib().oracle_ls_weights(C.c_int(ma.n_cells), _i(arrs[0]), _i(arrs[1]), _i(arrs[2]),
                            _i(arrs[3]), _d(arrs[4]), _d(arrs[5]), _d(arrs[6]), _d(arrs[7]),
                            _d(arrs[8]), C.c_int(mode), _d(lhs), _d(rhs))
    return lhs, rhs


class OracleRun:
    """A serial FP64 run of the reference time step on one case.

    ``cfg`` keys: visc, gamma, dt, domain_dt, pressure_gradient, channel_height,
    max_velocity, ref_rho, tolerance, origin, lengths, gradient_mode, and for
    the IBM: node_ref [N,3], node_x [N,3], stiffness, radius, depth,
    object_nodes.
    """

    def __init__(self, ma, rho_type, vel_type, bc_value, cfg, state0):
        self._keep = []
        self.ma = ma
        C_, F, B = ma.n_cells, ma.n_faces, ma.n_bc
        self.lhs, self.rhs = ls_weights(ma, int(cfg.get("gradient_mode", 0)))  # | 0x100: exact
        p = _Problem()
        p.n_cells, p.n_faces, p.n_internal = C_, F, ma.n_internal

        def keep(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a

        p.owner = _i(keep(ma.owner, np.int32))
        p.neighbour = _i(keep(ma.neighbour, np.int32))
        p.face_area = _d(keep(ma.face_area, np.float64))
        p.face_normal = _d(keep(ma.face_normal, np.float64))
        p.face_centroid = _d(keep(ma.face_centroid, np.float64))
        p.streaming_dt = _d(keep(ma.streaming_dt, np.float64))
        p.cell_volume = _d(keep(ma.cell_volume, np.float64))
        p.cell_centroid = _d(keep(ma.cell_centroid, np.float64))
        p.st_off = _i(keep(ma.stencil_offsets, np.int32))
        p.st_cells = _i(keep(ma.stencil_cells, np.int32))
        p.st_faces = _i(keep(ma.stencil_faces, np.int32))
        p.bc_rho_type = _i(keep(rho_type, np.int32))
        p.bc_vel_type = _i(keep(vel_type, np.int32))
        p.bc_value = _d(keep(bc_value, np.float64))
        p.lhs_inv = _d(keep(self.lhs, np.float64))
        p.rhs = _d(keep(self.rhs, np.float64))
        for k in ("visc", "gamma", "dt", "domain_dt", "pressure_gradient", "channel_height",
                  "max_velocity", "ref_rho", "tolerance"):
            setattr(p, k, float(cfg[k]))
        for a in range(3):
            p.origin[a] = float(cfg["origin"][a])
            p.lengths[a] = float(cfg["lengths"][a])
        node_ref = np.asarray(cfg.get("node_ref", np.zeros((0, 3))), np.float64).reshape(-1, 3)
        N = node_ref.shape[0]
        p.n_nodes = N
        p.object_nodes = int(cfg.get("object_nodes", max(N, 1)))
        p.node_ref = _d(keep(node_ref, np.float64))
        p.stiffness = float(cfg.get("stiffness", 0.0))
        p.radius = float(cfg.get("radius", 1.0))
        p.depth = float(cfg.get("depth", 1.0))
        p.flavour = int(cfg.get("flavour", 0))  # 1: the reference CPU Solver's tables
        self.p = p

        self.state = np.ascontiguousarray(state0, np.float64).reshape(C_ + B, 4).copy()
        self.t0 = np.zeros((C_, 4))
        self.t1 = np.zeros((C_, 4))
        nx = np.asarray(cfg.get("node_x", node_ref), np.float64).reshape(-1, 3)
        self.node_x = nx.copy()
        self.node_x0 = nx.copy()
        self.node_vel = np.zeros((N, 3))
        self.node_force = np.zeros((N, 3))
        self.force = np.zeros((C_, 3))
        self.grad = np.zeros((C_ + B, 12))
        self.face_flux = np.zeros((F, 4))
        self.residual = np.zeros((C_, 4))
        s = _State()
        s.state, s.t0, s.t1 = _d(self.state), _d(self.t0), _d(self.t1)
        s.node_x, s.node_x0 = _d(self.node_x), _d(self.node_x0)
        s.node_vel, s.node_force = _d(self.node_vel), _d(self.node_force)
        s.force, s.grad = _d(self.force), _d(self.grad)
        s.face_flux, s.residual = _d(self.face_flux), _d(self.residual)
        s.stage = 0
        self.s = s
        self.history = np.zeros((0, 6))
        lib().oracle_init_t1(C.byref(self.p), C.byref(self.s))

    def run_stages(self, n_stages, stop_on_convergence=False):
        hist = np.zeros((n_stages // 4 + 1, 6))
        self.s.history = _d(hist)
        steps = lib().oracle_run(C.byref(self.p), C.byref(self.s), int(n_stages),
                                 int(bool(stop_on_convergence)))
        self.history = np.concatenate([self.history, hist[:steps]])
        return steps

    def run_steps(self, n_steps, stop_on_convergence=False):
        return self.run_stages(4 * n_steps, stop_on_convergence)
