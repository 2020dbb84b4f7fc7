"""Learned warm start on the GPU: the mesh graph network's forward pass,
loss and every parameter gradient against the torch reference (CPU, same
BF16 rounding of the matrix-product operands), on a mesh graph whose row
counts are not multiples of the 128-row tiles, with both tensor-core paths
(mma.sync and tcgen05, forward and backward); the two paths against each
other on a graph with several tiles per block; and a short training run."""

import numpy as np
import pytest

from gnn_torch import TorchNet
from plfbs import cases, gnn

pytestmark = pytest.mark.gpu

NF, EF, OUT = 9, 4, 4


def _graph(nx=9, ny=7, nz=5):
    ma = cases.mesh_arrays(cases.uniform_box(nx, ny, nz), 0.01, 1.0, 1e-3)
    src, dst, ef = gnn.mesh_graph(ma)
    x = gnn.node_features(ma, (nx, ny, nz), (4.0, 3.5, 2.5), 3.0, 80.0)
    return ma, src, dst, ef, x


def _target(ma):
    c = np.asarray(ma.cell_centroid).reshape(-1, 3)[: ma.n_cells]
    return np.stack([np.sin(c[:, 0] / 3), np.cos(c[:, 1] / 2), c[:, 2] / 5 - 0.5,
                     0.1 * np.sin(c[:, 0] * c[:, 1] / 10)], 1).astype(np.float32)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("kind", [0, 1], ids=["mma_sync", "tcgen05"])
@pytest.mark.parametrize("layers", [1, 3])
def test_forward_loss_and_gradients_match_reference(plfbs_lib, layers, kind):
    ma, src, dst, ef, x = _graph()
    p = gnn.init_params(NF, EF, layers, OUT, seed=7, residual_scale=0.5)
    net = gnn.GraphNet(src, dst, ef, ma.n_cells, NF, layers, OUT)
    net.set_tensor_cores(kind)
    assert net.n_params == p.size
    net.set_params(p)
    np.testing.assert_array_equal(net.get_params(), p)
    ref = TorchNet(p, NF, EF, layers, OUT)
    y = net.forward(x)
    y_ref = ref.forward(x, ef, src, dst).detach().numpy()
    assert _rel(y, y_ref) < 5e-3
    t = _target(ma)
    loss, g = net.gradients(x, t)
    loss_ref, g_ref = ref.loss_and_grad(x, ef, src, dst, t)
    assert abs(loss - loss_ref) / loss_ref < 5e-3
    assert _rel(g, g_ref) < 3e-2
    # every MLP's block of parameters, not only the largest
    off = 0
    for k, o in gnn.mlp_sizes(NF, EF, layers, OUT):
        n = k * 64 + 64 + 64 * o + o
        assert _rel(g[off:off + n], g_ref[off:off + n]) < 6e-2, off
        off += n
    net.close()


def test_training_reduces_the_loss(plfbs_lib):
    ma, src, dst, ef, x = _graph()
    net = gnn.GraphNet(src, dst, ef, ma.n_cells, NF, 2, OUT)
    net.set_params(gnn.init_params(NF, EF, 2, OUT, seed=3))
    t = _target(ma)
    first = net.train_step(x, t, 2e-3)
    for _ in range(300):
        last = net.train_step(x, t, 2e-3)
    assert last < first / 10
    # deterministic: the same steps from the same start give the same bits
    net2 = gnn.GraphNet(src, dst, ef, ma.n_cells, NF, 2, OUT)
    net2.set_params(gnn.init_params(NF, EF, 2, OUT, seed=3))
    for _ in range(301):
        last2 = net2.train_step(x, t, 2e-3)
    assert last2 == last
    np.testing.assert_array_equal(net.get_params(), net2.get_params())


def test_tcgen05_forward_matches_mma_sync(plfbs_lib):
    """The two tensor-core paths take the same BF16 operands; their FP32 sums
    differ only in order. Larger graph: several 128-row tiles per block."""
    ma, src, dst, ef, x = _graph(24, 20, 18)
    p = gnn.init_params(NF, EF, 4, OUT, seed=5, residual_scale=0.5)
    net = gnn.GraphNet(src, dst, ef, ma.n_cells, NF, 4, OUT)
    net.set_params(p)
    net.set_tensor_cores(0)
    y0 = net.forward(x)
    net.set_tensor_cores(1)
    y1 = net.forward(x)
    y2 = net.forward(x)
    np.testing.assert_array_equal(y1, y2)  # deterministic
    assert _rel(y1, y0) < 2e-3
    with pytest.raises(gnn.GnnError):
        net.set_tensor_cores(2)


def test_tcgen05_gradients_match_mma_sync(plfbs_lib):
    """Forward and backward on tcgen05 against the mma.sync kernels: the same
    BF16 operands, FP32 sums in another order; every MLP's gradient block,
    deterministic from run to run. Several 128-row tiles per block, so the
    weight gradients accumulate in tensor memory over tiles."""
    ma, src, dst, ef, x = _graph(24, 20, 18)
    p = gnn.init_params(NF, EF, 3, OUT, seed=11, residual_scale=0.5)
    net = gnn.GraphNet(src, dst, ef, ma.n_cells, NF, 3, OUT)
    net.set_params(p)
    t = _target(ma)
    net.set_tensor_cores(0)
    loss0, g0 = net.gradients(x, t)
    net.set_tensor_cores(1)
    loss1, g1 = net.gradients(x, t)
    loss2, g2 = net.gradients(x, t)
    net.close()
    np.testing.assert_array_equal(g1, g2)
    assert loss1 == loss2
    assert abs(loss1 - loss0) / loss0 < 1e-3
    assert _rel(g1, g0) < 5e-3
    off = 0
    for k, o in gnn.mlp_sizes(NF, EF, 3, OUT):
        n = k * 64 + 64 + 64 * o + o
        assert _rel(g1[off:off + n], g0[off:off + n]) < 2e-2, off
        off += n
