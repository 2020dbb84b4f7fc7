"""Learned warm start: ctypes binding of include/plfbs_gnn.h plus the graph,
feature and parameter builders for a mesh.

The graph is the solver's own face connectivity: two directed edges per
internal face between its owner and neighbour cells. Node features are the
cell centroid (scaled to the box), the signed distance to the sphere surface
in diameters, 1 / (1 + that distance^2) and Re / 200; edge features are the
centroid offset and its length.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)

HIDDEN = 64

EXPORTS = ("plfbs_gnn_create", "plfbs_gnn_param_count", "plfbs_gnn_set_params",
           "plfbs_gnn_get_params", "plfbs_gnn_forward", "plfbs_gnn_gradients",
           "plfbs_gnn_train_step", "plfbs_gnn_last_error", "plfbs_gnn_destroy",
           "plfbs_gnn_set_tensor_cores")


class Shape(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("n_edges", C.c_int32), ("node_features", C.c_int32),
                ("edge_features", C.c_int32), ("layers", C.c_int32), ("outputs", C.c_int32)]


_bound = False


def lib():
    global _bound
    L = capi.lib()
    if not _bound:
        L.plfbs_gnn_create.argtypes = [C.POINTER(Shape), _ip, _ip, _fp, C.c_int32,
                                       C.POINTER(C.c_void_p)]
        L.plfbs_gnn_param_count.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        L.plfbs_gnn_set_params.argtypes = [C.c_void_p, _fp, C.c_int64]
        L.plfbs_gnn_get_params.argtypes = [C.c_void_p, _fp, C.c_int64]
        L.plfbs_gnn_forward.argtypes = [C.c_void_p, _fp, _fp]
        L.plfbs_gnn_gradients.argtypes = [C.c_void_p, _fp, _fp, C.POINTER(C.c_double), _fp]
        L.plfbs_gnn_train_step.argtypes = [C.c_void_p, _fp, _fp, C.c_float,
                                           C.POINTER(C.c_double)]
        L.plfbs_gnn_last_error.argtypes = [C.c_void_p]
        L.plfbs_gnn_last_error.restype = C.c_char_p
        L.plfbs_gnn_destroy.argtypes = [C.c_void_p]
        L.plfbs_gnn_set_tensor_cores.argtypes = [C.c_void_p, C.c_int32]
        _bound = True
    return L


def _f(a):
    return a.ctypes.data_as(_fp)


def mlp_sizes(node_features, edge_features, layers, outputs):
    """(kin, out) of every MLP in the flat parameter order."""
    s = [(node_features, HIDDEN), (edge_features, HIDDEN)]
    for _ in range(layers):
        s += [(3 * HIDDEN, HIDDEN), (2 * HIDDEN, HIDDEN)]
    s.append((HIDDEN, outputs))
    return s


def param_count(node_features, edge_features, layers, outputs):
    return sum(k * HIDDEN + HIDDEN + HIDDEN * o + o
               for k, o in mlp_sizes(node_features, edge_features, layers, outputs))


def init_params(node_features, edge_features, layers, outputs, seed=0, residual_scale=0.1):
    """He-normal first layers, small second layers in the residual MLPs."""
    rng = np.random.default_rng(seed)
    out = []
    sizes = mlp_sizes(node_features, edge_features, layers, outputs)
    for i, (k, o) in enumerate(sizes):
        w1 = rng.normal(0.0, np.sqrt(2.0 / k), (k, HIDDEN))
        scale = residual_scale if 2 <= i < len(sizes) - 1 else 1.0
        w2 = rng.normal(0.0, scale * np.sqrt(1.0 / HIDDEN), (HIDDEN, o))
        out += [w1.ravel(), np.zeros(HIDDEN), w2.ravel(), np.zeros(o)]
    return np.concatenate(out).astype(np.float32)


def mesh_graph(ma):
    """Directed edges (both ways per internal face) and edge features
    (centroid offset dx, dy, dz and its length) of a solver mesh."""
    fi = ma.n_internal
    o = np.asarray(ma.owner[:fi], np.int32)
    n = np.asarray(ma.neighbour[:fi], np.int32)
    src = np.concatenate([o, n]).astype(np.int32)
    dst = np.concatenate([n, o]).astype(np.int32)
    c = np.asarray(ma.cell_centroid, np.float64).reshape(-1, 3)
    d = c[dst] - c[src]
    feat = np.concatenate([d, np.linalg.norm(d, axis=1, keepdims=True)], axis=1)
    return src, dst, feat.astype(np.float32)


def node_features(ma, lengths, centre, diameter, re, relative=True):
    """[n_cells][9]: x, y, z / box lengths, signed distance to the sphere in
    diameters, 1 / (1 + that^2), Re / 200 and, with `relative`, the offset from
    the sphere centre in units of 4 diameters (which side of the sphere a cell
    lies on: a cell downstream sits in the wake); [n_cells][6] without."""
    c = np.asarray(ma.cell_centroid, np.float64).reshape(-1, 3)[: ma.n_cells]
    d = c - np.asarray(centre, np.float64)
    sd = (np.linalg.norm(d, axis=1) - diameter / 2) / diameter
    f = np.empty((ma.n_cells, 9 if relative else 6))
    f[:, :3] = c / np.asarray(lengths, np.float64)
    f[:, 3] = sd
    f[:, 4] = 1.0 / (1.0 + sd * sd)
    f[:, 5] = re / 200.0
    if relative:
        f[:, 6:9] = d / (4.0 * diameter)
    return f.astype(np.float32)


class GnnError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("plfbs_gnn error %d: %s" % (code, message))
        self.code = code


class GraphNet:
    """The network on one GPU; all arrays are host numpy float32."""

    def __init__(self, src, dst, edge_features, n_nodes, node_features, layers, outputs,
                 device=0):
        L = lib()
        self.src = np.ascontiguousarray(src, np.int32)
        self.dst = np.ascontiguousarray(dst, np.int32)
        ef = np.ascontiguousarray(edge_features, np.float32)
        self.shape = Shape(int(n_nodes), len(self.src), int(node_features), ef.shape[1],
                           int(layers), int(outputs))
        h = C.c_void_p()
        rc = L.plfbs_gnn_create(C.byref(self.shape), self.src.ctypes.data_as(_ip),
                                self.dst.ctypes.data_as(_ip), _f(ef), int(device), C.byref(h))
        if rc:
            raise GnnError(rc, L.plfbs_gnn_last_error(None).decode())
        self.h = h
        n = C.c_int64()
        self._check(L.plfbs_gnn_param_count(self.h, C.byref(n)))
        self.n_params = n.value

    def _check(self, rc):
        if rc:
            raise GnnError(rc, lib().plfbs_gnn_last_error(self.h).decode())

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(lib().plfbs_gnn_set_params(self.h, _f(p), p.size))

    def get_params(self):
        p = np.zeros(self.n_params, np.float32)
        self._check(lib().plfbs_gnn_get_params(self.h, _f(p), p.size))
        return p

    def set_tensor_cores(self, kind):
        """1: tcgen05 forward (the default), 0: mma.sync forward."""
        self._check(lib().plfbs_gnn_set_tensor_cores(self.h, int(kind)))

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((self.shape.n_nodes, self.shape.outputs), np.float32)
        self._check(lib().plfbs_gnn_forward(self.h, _f(x), _f(y)))
        return y

    def gradients(self, x, target):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_double()
        self._check(lib().plfbs_gnn_gradients(self.h, _f(x), _f(t), C.byref(loss), _f(g)))
        return loss.value, g

    def train_step(self, x, target, lr):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        loss = C.c_double()
        self._check(lib().plfbs_gnn_train_step(self.h, _f(x), _f(t), float(lr), C.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            lib().plfbs_gnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def main(argv=None):
    """Times training steps of the network (forward, backward, Adam) on the
    face graph of the warm start's 64 x 32 x 32 channel (65,536 nodes, 8
    message-passing layers, 9 node / 4 edge features, 4 outputs) with seeded
    synthetic features and targets; prints one JSON line. The command behind
    the committed ncu summary of the network's kernels:

        python -m plfbs.gnn --steps 5 [--tensor-cores 0|1]
    """
    import argparse
    import json
    import time

    from . import cases
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--tensor-cores", type=int, default=1)
    args = ap.parse_args(argv)
    ma = cases.mesh_arrays(cases.uniform_box(64, 32, 32), 0.008, 1.0, 0.0)
    src, dst, ef = mesh_graph(ma)
    x = node_features(ma, (64, 32, 32), (16.0, 16.0, 16.0), 8.0, 100.0)
    rng = np.random.Generator(np.random.PCG64(0))
    t = rng.standard_normal((ma.n_cells, 4)).astype(np.float32)
    net = GraphNet(src, dst, ef, ma.n_cells, x.shape[1], 8, 4)
    net.set_params(init_params(x.shape[1], ef.shape[1], 8, 4, seed=1))
    net.set_tensor_cores(args.tensor_cores)
    net.train_step(x, t, 1e-4)  # warm-up
    t0 = time.perf_counter()
    losses = [net.train_step(x, t, 1e-4) for _ in range(args.steps)]
    dt = (time.perf_counter() - t0) / max(args.steps, 1)
    t1 = time.perf_counter()
    net.forward(x)
    fwd = time.perf_counter() - t1
    net.close()
    print(json.dumps({"graph_nodes": int(ma.n_cells), "graph_edges": int(len(src)), "layers": 8,
                      "train_step_s": dt, "forward_s": fwd, "loss_first": losses[0],
                      "loss_last": losses[-1], "tensor_cores": args.tensor_cores}))


if __name__ == "__main__":
    main()
