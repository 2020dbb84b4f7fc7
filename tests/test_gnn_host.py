"""Learned warm start, host side: graph and feature builders, parameter
layout, and the torch reference model used as the GPU kernels' oracle."""

import numpy as np

from gnn_torch import TorchNet
from plfbs import cases, gnn


def _small_mesh(nx=6, ny=5, nz=4):
    pm = cases.uniform_box(nx, ny, nz)
    return cases.mesh_arrays(pm, 0.01, 1.0, 1e-3)


def test_graph_has_two_edges_per_internal_face():
    ma = _small_mesh()
    src, dst, ef = gnn.mesh_graph(ma)
    assert len(src) == 2 * ma.n_internal
    assert src.max() < ma.n_cells and dst.max() < ma.n_cells
    pairs = set(zip(src.tolist(), dst.tolist()))
    assert all((d, s) in pairs for s, d in pairs)  # both directions
    np.testing.assert_allclose(ef[:, 3], 1.0)  # unit spacing
    np.testing.assert_allclose(np.abs(ef[:, :3]).sum(1), 1.0)


def test_node_features():
    ma = _small_mesh()
    f = gnn.node_features(ma, (6, 5, 4), (3.0, 2.5, 2.0), 2.0, 100.0)
    assert f.shape == (ma.n_cells, 9) and f.dtype == np.float32
    assert f[:, 3].min() < 0 < f[:, 3].max()  # cells inside and outside the sphere
    np.testing.assert_allclose(f[:, 5], 0.5)
    c = np.asarray(ma.cell_centroid).reshape(-1, 3)[: ma.n_cells]
    np.testing.assert_allclose(f[:, 6:9], (c - [3.0, 2.5, 2.0]) / 8.0, rtol=1e-6)
    f6 = gnn.node_features(ma, (6, 5, 4), (3.0, 2.5, 2.0), 2.0, 100.0, relative=False)
    np.testing.assert_array_equal(f6, f[:, :6])


def test_param_layout_and_reference_model():
    nf, ef_, L, out = 9, 4, 2, 4
    p = gnn.init_params(nf, ef_, L, out, seed=1)
    assert p.size == gnn.param_count(nf, ef_, L, out)
    ma = _small_mesh()
    src, dst, ef = gnn.mesh_graph(ma)
    x = gnn.node_features(ma, (6, 5, 4), (3.0, 2.5, 2.0), 2.0, 100.0)
    net = TorchNet(p, nf, ef_, L, out)
    y16 = net.forward(x, ef, src, dst, bf16=True).detach().numpy()
    y32 = net.forward(x, ef, src, dst, bf16=False).detach().numpy()
    assert y16.shape == (ma.n_cells, out)
    rel = np.linalg.norm(y16 - y32) / np.linalg.norm(y32)
    assert 0 < rel < 3e-2  # BF16 operands, FP32 sums
    loss, g = net.loss_and_grad(x, ef, src, dst, np.zeros_like(y16))
    assert g.shape == p.shape and np.isfinite(g).all() and loss > 0
