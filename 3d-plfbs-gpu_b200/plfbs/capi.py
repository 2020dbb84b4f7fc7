"""ctypes binding of include/plfbs.h (libplfbs.so) and a small Python front end.

This is the Python view of the same C ABI the reference-side C++ shim uses; it
loads the in-tree library and raises if it is missing (no fallback path).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "libplfbs.so")

OK, ERR_ARG, ERR_MESH, ERR_BC, ERR_CUDA, ERR_DIVERGED, ERR_NO_DEVICE, ERR_STATE, ERR_TIMEOUT = (
    0, -1, -2, -3, -4, -5, -6, -7, -8)
GRAD_LS, GRAD_HYBRID, GRAD_GREEN_GAUSS, GRAD_EXACT_INVERSE = 0, 1, 2, 0x100
FP64, FP32_DEVIATION = 0, 1
FLAVOUR_GPU, FLAVOUR_CPU_SOLVER = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)

# every symbol include/plfbs.h declares
EXPORTS = ("plfbs_create", "plfbs_set_state", "plfbs_run", "plfbs_get_state",
           "plfbs_get_nodes", "plfbs_get_body_force", "plfbs_set_debug", "plfbs_run_stages",
           "plfbs_get_gradients", "plfbs_get_face_flux", "plfbs_get_residual",
           "plfbs_ls_weights", "plfbs_profile_steps", "plfbs_memory_bytes",
           "plfbs_last_error", "plfbs_destroy", "plfbs_version",
           "plfbs_residual_norms_noalloc", "plfbs_release_cached", "plfbs_warm_start",
           "plfbs_checkpoint_bytes", "plfbs_save_checkpoint", "plfbs_load_checkpoint",
           "plfbs_wall_forces", "plfbs_get_layout", "plfbs_polymesh_geometry",
           "plfbs_set_flux_kernel", "plfbs_set_layout_compression", "plfbs_cell_order",
           "plfbs_set_timeout", "plfbs_wait", "plfbs_profile_kernels", "plfbs_fp64_fma_peak")


class MeshView(C.Structure):
    _fields_ = [("n_cells", C.c_int32), ("n_faces", C.c_int32), ("n_internal", C.c_int32),
                ("owner", _ip), ("neighbour", _ip), ("face_area", _dp), ("face_normal", _dp),
                ("face_centroid", _dp), ("streaming_dt", _dp), ("cell_volume", _dp),
                ("cell_centroid", _dp), ("stencil_offsets", _ip), ("stencil_cells", _ip),
                ("stencil_faces", _ip)]


class PolyMeshView(C.Structure):
    _fields_ = [("n_points", C.c_int32), ("n_faces", C.c_int32), ("n_internal", C.c_int32),
                ("n_cells", C.c_int32), ("points", C.POINTER(C.c_float)),
                ("face_offsets", _ip), ("face_points", _ip), ("owner", _ip), ("neighbour", _ip)]


class MeshOut(C.Structure):
    _fields_ = [("owner", _ip), ("neighbour", _ip), ("face_area", _dp), ("face_normal", _dp),
                ("face_centroid", _dp), ("streaming_dt", _dp), ("cell_volume", _dp),
                ("cell_centroid", _dp), ("stencil_offsets", _ip), ("stencil_cells", _ip),
                ("stencil_faces", _ip)]


class BCView(C.Structure):
    _fields_ = [("rho_type", _ip), ("vel_type", _ip), ("value", _dp)]


class IBMView(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("x_ref", _dp), ("x", _dp), ("stiffness", C.c_double),
                ("radius", C.c_double), ("depth", C.c_double), ("object_nodes", C.c_int32)]


class Config(C.Structure):
    _fields_ = [("visc", C.c_double), ("gamma", C.c_double), ("time_marching_step", C.c_double),
                ("domain_dt", C.c_double), ("max_velocity", C.c_double), ("ref_rho", C.c_double),
                ("tolerance", C.c_double), ("pressure_gradient", C.c_double),
                ("channel_height", C.c_double), ("origin", C.c_double * 3),
                ("lengths", C.c_double * 3), ("gradient_mode", C.c_int32),
                ("precision", C.c_int32), ("renumber", C.c_int32), ("flavour", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("steps_done", C.c_int64), ("converged", C.c_int32), ("status", C.c_int32),
                ("max_error", C.c_double), ("rho_rms", C.c_double), ("u_rms", C.c_double),
                ("v_rms", C.c_double), ("w_rms", C.c_double), ("kernel_ms", C.c_double),
                ("steps_run", C.c_int64)]


_lib = None


def lib():
    """Load libplfbs.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libplfbs.so is missing at %s: run `python -m plfbs.build`"
                               % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        L.plfbs_last_error.restype = C.c_char_p
        L.plfbs_version.restype = C.c_char_p
        L.plfbs_create.argtypes = [C.POINTER(Config), C.POINTER(MeshView), C.POINTER(BCView),
                                   C.POINTER(IBMView), C.c_int, C.POINTER(C.c_void_p)]
        for name in ("plfbs_set_state", "plfbs_get_state"):
            getattr(L, name).argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.c_int64]
        L.plfbs_run.argtypes = [C.c_void_p, C.c_int64, C.POINTER(Stats), _dp]
        L.plfbs_get_nodes.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int32]
        L.plfbs_get_body_force.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
        L.plfbs_set_debug.argtypes = [C.c_void_p, C.c_int]
        L.plfbs_run_stages.argtypes = [C.c_void_p, C.c_int64]
        for name in ("plfbs_get_gradients", "plfbs_get_face_flux", "plfbs_get_residual"):
            getattr(L, name).argtypes = [C.c_void_p, _dp, C.c_int32]
        L.plfbs_ls_weights.argtypes = [C.POINTER(MeshView), C.c_int32, _dp, _dp]
        L.plfbs_profile_steps.argtypes = [C.c_void_p, C.c_int64, _dp]
        L.plfbs_profile_kernels.argtypes = [C.c_void_p, C.c_int64, _dp]
        L.plfbs_fp64_fma_peak.argtypes = [C.c_int32, _dp]
        L.plfbs_memory_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        L.plfbs_last_error.argtypes = [C.c_void_p]
        L.plfbs_destroy.argtypes = [C.c_void_p]
        L.plfbs_release_cached.argtypes = [C.c_int32]
        L.plfbs_warm_start.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.c_int64, _dp, C.c_int32]
        L.plfbs_checkpoint_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        L.plfbs_wall_forces.argtypes = [C.c_void_p, _ip, C.c_int32, _dp, _dp]
        L.plfbs_get_layout.argtypes = [C.c_void_p, _ip, _ip, _ip, _ip, _dp, _ip]
        L.plfbs_set_flux_kernel.argtypes = [C.c_void_p, C.c_int32]
        L.plfbs_set_layout_compression.argtypes = [C.c_void_p, C.c_int32]
        L.plfbs_set_timeout.argtypes = [C.c_void_p, C.c_double]
        L.plfbs_wait.argtypes = [C.c_void_p, C.c_double]
        L.plfbs_cell_order.argtypes = [C.POINTER(MeshView), C.c_int32, _ip]
        L.plfbs_polymesh_geometry.argtypes = [C.POINTER(PolyMeshView), C.c_double, C.c_double,
                                              C.c_double, C.c_int32, C.POINTER(MeshOut)]
        L.plfbs_save_checkpoint.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        L.plfbs_load_checkpoint.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        L.plfbs_release_cached.restype = C.c_int
        L.plfbs_residual_norms_noalloc.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.c_double,
                                                   C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


class PlfbsError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("plfbs error %d: %s" % (code, message))
        self.code = code


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def mesh_view(ma, keep):
    """A MeshView over the arrays of a cases.MeshArrays (kept alive in ``keep``)."""
    def k(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a
    v = MeshView()
    v.n_cells, v.n_faces, v.n_internal = ma.n_cells, ma.n_faces, ma.n_internal
    v.owner = _i(k(ma.owner, np.int32))
    v.neighbour = _i(k(ma.neighbour, np.int32))
    v.face_area = _d(k(ma.face_area, np.float64))
    v.face_normal = _d(k(ma.face_normal, np.float64))
    v.face_centroid = _d(k(ma.face_centroid, np.float64))
    v.streaming_dt = _d(k(ma.streaming_dt, np.float64))
    v.cell_volume = _d(k(ma.cell_volume, np.float64))
    v.cell_centroid = _d(k(ma.cell_centroid, np.float64))
    v.stencil_offsets = _i(k(ma.stencil_offsets, np.int32))
    v.stencil_cells = _i(k(ma.stencil_cells, np.int32))
    v.stencil_faces = _i(k(ma.stencil_faces, np.int32))
    return v


def fp64_fma_peak(device=0):
    """Measured FP64 FMA throughput of a device in GFLOP/s (plfbs_fp64_fma_peak)."""
    g = C.c_double()
    rc = lib().plfbs_fp64_fma_peak(int(device), C.byref(g))
    if rc:
        raise PlfbsError(rc, lib().plfbs_last_error(None).decode())
    return g.value


def cell_order(ma, renumber):
    """Host-only: the cell order plfbs_create uses (order[new] = caller cell)."""
    keep = []
    v = mesh_view(ma, keep)
    order = np.zeros(ma.n_cells, np.int32)
    rc = lib().plfbs_cell_order(C.byref(v), int(renumber), _i(order))
    if rc:
        raise PlfbsError(rc, lib().plfbs_last_error(None).decode())
    return order


def ls_weights(ma, mode):
    """Host-only least-squares weights: (lhs_inv [C,3,3], rhs [nnz,3])."""
    keep = []
    v = mesh_view(ma, keep)
    nnz = int(ma.stencil_offsets[-1])
    lhs = np.zeros((ma.n_cells, 3, 3))
    rhs = np.zeros((nnz, 3))
    rc = lib().plfbs_ls_weights(C.byref(v), int(mode), _d(lhs), _d(rhs))
    if rc:
        raise PlfbsError(rc, lib().plfbs_last_error(None).decode())
    return lhs, rhs


def polymesh_geometry(pm, visc, gamma, fneq_min, device=0):
    """The solver's mesh arrays (a cases.MeshArrays) of a cases.PolyMesh,
    computed on the GPU by plfbs_polymesh_geometry."""
    from . import cases
    F, Fi, Cn = pm.n_faces, pm.n_internal, pm.n_cells
    B = F - Fi
    nv = np.asarray(pm.nverts, np.int32)
    offsets = np.zeros(F + 1, np.int32)
    np.cumsum(nv, out=offsets[1:])
    faces = np.asarray(pm.faces)
    fp = np.ascontiguousarray(faces[np.arange(faces.shape[1])[None, :] < nv[:, None]], np.int32)
    pts = np.ascontiguousarray(pm.points, np.float32)
    owner = np.ascontiguousarray(pm.owner, np.int32)
    nb = np.ascontiguousarray(pm.neighbour, np.int32)
    v = PolyMeshView()
    v.n_points, v.n_faces, v.n_internal, v.n_cells = pts.shape[0], F, Fi, Cn
    v.points = pts.ctypes.data_as(C.POINTER(C.c_float))
    v.face_offsets, v.face_points, v.owner, v.neighbour = _i(offsets), _i(fp), _i(owner), _i(nb)
    T, nnz = Cn + B, 2 * Fi + B
    a = dict(owner=np.zeros(F, np.int32), neighbour=np.zeros(F, np.int32),
             face_area=np.zeros(F), face_normal=np.zeros((F, 3)), face_centroid=np.zeros((F, 3)),
             streaming_dt=np.zeros(F), cell_volume=np.zeros(T), cell_centroid=np.zeros((T, 3)),
             stencil_offsets=np.zeros(Cn + 1, np.int32), stencil_cells=np.zeros(nnz, np.int32),
             stencil_faces=np.zeros(nnz, np.int32))
    o = MeshOut()
    for k, arr in a.items():
        setattr(o, k, _i(arr) if arr.dtype == np.int32 else _d(arr))
    rc = lib().plfbs_polymesh_geometry(C.byref(v), float(visc), float(gamma), float(fneq_min),
                                       int(device), C.byref(o))
    if rc:
        raise PlfbsError(rc, lib().plfbs_last_error(None).decode())
    return cases.MeshArrays(n_cells=Cn, n_faces=F, n_internal=Fi, bc_types=pm.bc_types(), **a)


class Solver:
    """One plfbs context on one GPU.

    ``cfg`` keys: visc, gamma, dt (time_marching_step), domain_dt, max_velocity,
    ref_rho, tolerance, pressure_gradient, channel_height, origin, lengths,
    gradient_mode, precision (FP64 or FP32_DEVIATION), renumber (0 the mesh's
    cell order, 1 reverse Cuthill-McKee on the host, 2 the same order built on
    the device), flavour (FLAVOUR_GPU or FLAVOUR_CPU_SOLVER). ``ibm``
    (optional): node_ref [N,3], node_x [N,3], stiffness, radius, depth,
    object_nodes.
    """

    def __init__(self, ma, rho_type, vel_type, bc_value, cfg, ibm=None, device=0):
        self._keep = []
        self.ma = ma
        self.C, self.F, self.B = ma.n_cells, ma.n_faces, ma.n_bc
        self.T = self.C + self.B
        L = lib()
        mv = mesh_view(ma, self._keep)
        bv = BCView()
        rt = np.ascontiguousarray(rho_type, np.int32)
        vt = np.ascontiguousarray(vel_type, np.int32)
        bval = np.ascontiguousarray(bc_value, np.float64).reshape(-1, 4)
        self._keep += [rt, vt, bval]
        bv.rho_type, bv.vel_type, bv.value = _i(rt), _i(vt), _d(bval)
        cf = Config()
        cf.visc = cfg["visc"]
        cf.gamma = cfg.get("gamma", 1.0)
        cf.time_marching_step = cfg["dt"]
        cf.domain_dt = cfg.get("domain_dt", 0.5)
        cf.max_velocity = cfg["max_velocity"]
        cf.ref_rho = cfg.get("ref_rho", 1.0)
        cf.tolerance = cfg.get("tolerance", 0.0)
        cf.pressure_gradient = cfg.get("pressure_gradient", 0.0)
        cf.channel_height = cfg.get("channel_height", 1.0)
        for a in range(3):
            cf.origin[a] = cfg.get("origin", (0.0, 0.0, 0.0))[a]
            cf.lengths[a] = cfg.get("lengths", (1.0, 1.0, 1.0))[a]
        cf.gradient_mode = cfg.get("gradient_mode", GRAD_LS)
        cf.precision = cfg.get("precision", FP64)
        cf.renumber = cfg.get("renumber", 0)
        cf.flavour = cfg.get("flavour", FLAVOUR_GPU)
        iv = IBMView()
        self.N = 0
        if ibm is not None and len(ibm.get("node_ref", [])) > 0:
            nref = np.ascontiguousarray(ibm["node_ref"], np.float64).reshape(-1, 3)
            nx = np.ascontiguousarray(ibm.get("node_x", nref), np.float64).reshape(-1, 3)
            self._keep += [nref, nx]
            self.N = nref.shape[0]
            iv.n_nodes = self.N
            iv.x_ref, iv.x = _d(nref), _d(nx)
            iv.stiffness = ibm.get("stiffness", 0.0)
            iv.radius = ibm.get("radius", 1.0)
            iv.depth = ibm.get("depth", 1.0)
            iv.object_nodes = int(ibm.get("object_nodes", self.N))
        h = C.c_void_p()
        rc = L.plfbs_create(C.byref(cf), C.byref(mv), C.byref(bv), C.byref(iv), int(device),
                            C.byref(h))
        if rc:
            raise PlfbsError(rc, L.plfbs_last_error(None).decode())
        self.h = h
        self._keep.clear()

    def _check(self, rc):
        if rc:
            raise PlfbsError(rc, lib().plfbs_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().plfbs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, state):
        """state [C+B, 4] = (u, v, w, rho) in caller numbering."""
        s = np.asarray(state, np.float64).reshape(self.T, 4)
        cols = [np.ascontiguousarray(s[:, k]) for k in (3, 0, 1, 2)]
        self._check(lib().plfbs_set_state(self.h, *[_d(c) for c in cols], self.T))

    def get_state(self):
        cols = [np.zeros(self.T) for _ in range(4)]
        self._check(lib().plfbs_get_state(self.h, *[_d(c) for c in cols], self.T))
        rho, u, v, w = cols
        return np.stack([u, v, w, rho], axis=1)

    def set_fields(self, rho, u, v, w):
        """The state from four caller arrays of C+B FP64 values, passed to
        plfbs_set_state as they are (pinned host memory copies at the copy
        engines' rate)."""
        cols = (rho, u, v, w)
        for c in cols:
            if not (isinstance(c, np.ndarray) and c.dtype == np.float64 and c.size == self.T
                    and c.flags.c_contiguous):
                raise ValueError("set_fields needs contiguous float64 arrays of C+B values")
        self._check(lib().plfbs_set_state(self.h, *[_d(c) for c in cols], self.T))

    def get_fields(self, rho, u, v, w):
        """plfbs_get_state into four caller arrays of C+B FP64 values."""
        cols = (rho, u, v, w)
        for c in cols:
            if not (isinstance(c, np.ndarray) and c.dtype == np.float64 and c.size == self.T
                    and c.flags.c_contiguous and c.flags.writeable):
                raise ValueError("get_fields needs writable contiguous float64 arrays")
        self._check(lib().plfbs_get_state(self.h, *[_d(c) for c in cols], self.T))

    def run(self, max_steps, history=True):
        st = Stats()
        hist = np.zeros((max(int(max_steps), 1), 6)) if history else None
        rc = lib().plfbs_run(self.h, int(max_steps), C.byref(st),
                             _d(hist) if history else C.cast(None, _dp))
        out = {k: getattr(st, k) for k, _ in Stats._fields_}
        if rc and rc != ERR_DIVERGED:
            self._check(rc)
        out["rc"] = rc
        return out, (hist[: int(st.steps_run)] if history else None)

    def set_timeout(self, seconds):
        """Bound plfbs_run's wait per batch of launched steps (0: no bound)."""
        self._check(lib().plfbs_set_timeout(self.h, float(seconds)))

    def wait(self, seconds):
        """True once the steps of a timed-out run have ended, False if they are
        still in flight after `seconds`."""
        rc = lib().plfbs_wait(self.h, float(seconds))
        if rc == ERR_TIMEOUT:
            return False
        self._check(rc)
        return True

    def run_stages(self, n):
        self._check(lib().plfbs_run_stages(self.h, int(n)))

    def set_debug(self, on=True):
        self._check(lib().plfbs_set_debug(self.h, int(bool(on))))

    def gradients(self):
        g = np.zeros((self.C, 12))
        self._check(lib().plfbs_get_gradients(self.h, _d(g), self.C))
        return g

    def face_flux(self):
        g = np.zeros((self.F, 4))
        self._check(lib().plfbs_get_face_flux(self.h, _d(g), self.F))
        return g

    def residual(self):
        g = np.zeros((self.C, 4))
        self._check(lib().plfbs_get_residual(self.h, _d(g), self.C))
        return g

    def warm_start(self, state, node_x=None):
        """Start from `state` [T, 4] (u, v, w, rho) with conserved RK seeding and,
        optionally, IBM node positions [N, 3]."""
        q = np.ascontiguousarray(state, np.float64).reshape(self.T, 4)
        cols = [np.ascontiguousarray(q[:, k]) for k in (3, 0, 1, 2)]
        nx = None
        if node_x is not None:
            nx = np.ascontiguousarray(node_x, np.float64).reshape(self.N, 3)
        self._check(lib().plfbs_warm_start(self.h, *[_d(c) for c in cols], self.T,
                                           _d(nx) if nx is not None else None, self.N))

    def set_flux_kernel(self, kind):
        """0: one thread per face (default); 1: TMA-staged internal faces (FP64;
        both give the same bits)."""
        self._check(lib().plfbs_set_flux_kernel(self.h, int(kind)))

    def set_layout_compression(self, on):
        """1: the kernels read the deduplicated record tables (FP64, default where
        available); 0: the per-face / per-cell arrays."""
        self._check(lib().plfbs_set_layout_compression(self.h, int(bool(on))))

    def layout(self):
        """The device-built layout (device numbering): dict of cell_order [C],
        face_order [F], stencil_nbr [K, C], stencil_w [3, K, C], gather [K2, C],
        compact = (unique face records, unique cell weight sets) in use."""
        sz = np.zeros(4, np.int32)
        self._check(lib().plfbs_get_layout(self.h, _i(sz), None, None, None, None, None))
        K, K2 = int(sz[0]), int(sz[1])
        out = dict(cell_order=np.zeros(self.C, np.int32), face_order=np.zeros(self.F, np.int32),
                   stencil_nbr=np.zeros((K, self.C), np.int32),
                   stencil_w=np.zeros((3, K, self.C)), gather=np.zeros((K2, self.C), np.int32))
        self._check(lib().plfbs_get_layout(self.h, _i(sz), _i(out["cell_order"]),
                                           _i(out["face_order"]), _i(out["stencil_nbr"]),
                                           _d(out["stencil_w"]), _i(out["gather"])))
        out["compact"] = (int(sz[2]), int(sz[3]))
        return out

    def wall_forces(self, wall_bc):
        """(Cd, Cl) over the boundary faces `wall_bc` (caller numbering)."""
        w = np.ascontiguousarray(wall_bc, np.int32)
        cd, cl = C.c_double(), C.c_double()
        self._check(lib().plfbs_wall_forces(self.h, _i(w), len(w), C.byref(cd), C.byref(cl)))
        return cd.value, cl.value

    def checkpoint(self):
        """The context's lossless checkpoint image (bytes)."""
        n = C.c_int64()
        self._check(lib().plfbs_checkpoint_bytes(self.h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        self._check(lib().plfbs_save_checkpoint(self.h, buf, n.value))
        return buf.raw

    def restore(self, image):
        self._check(lib().plfbs_load_checkpoint(self.h, image, len(image)))

    def nodes(self):
        x, v, f = (np.zeros((self.N, 3)) for _ in range(3))
        self._check(lib().plfbs_get_nodes(self.h, _d(x), _d(v), _d(f), self.N))
        return x, v, f

    def body_force(self, frontal_area):
        cd, cl = C.c_double(), C.c_double()
        self._check(lib().plfbs_get_body_force(self.h, float(frontal_area), C.byref(cd),
                                               C.byref(cl)))
        return cd.value, cl.value

    def profile_steps(self, n):
        ms = np.zeros(4)
        self._check(lib().plfbs_profile_steps(self.h, int(n), _d(ms)))
        return dict(zip(("ibm", "gradient", "flux", "update"), ms.tolist()))

    def profile_kernels(self, launches):
        """Mean device milliseconds per launch of each kernel kind, launched
        back to back (plfbs_profile_kernels); the run is left as it was."""
        ms = np.zeros(5)
        self._check(lib().plfbs_profile_kernels(self.h, int(launches), _d(ms)))
        return dict(zip(("ibm", "gradient", "flux", "update", "finish"), ms.tolist()))

    def memory_bytes(self):
        b = C.c_int64()
        self._check(lib().plfbs_memory_bytes(self.h, C.byref(b)))
        return b.value
