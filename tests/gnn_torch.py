"""Reference of the learned warm-start network in torch (CPU, FP32): the
oracle for the GPU kernels of csrc/gnn.cu. Test infrastructure only.

Mirrors include/plfbs_gnn.h: every MLP is Linear(k, 64) -> ReLU ->
Linear(64, m); the inputs of both matrix products are rounded to BF16 (as
the kernels stage them for the tensor cores) while sums, biases, residuals
and aggregates stay FP32. With bf16=False the model is plain FP32.
"""

import numpy as np
import torch

HIDDEN = 64


def _r(x, bf16):
    return x.to(torch.bfloat16).to(torch.float32) if bf16 else x


class TorchNet:
    def __init__(self, params, node_features, edge_features, layers, outputs):
        self.kin = [node_features, edge_features] + [3 * HIDDEN, 2 * HIDDEN] * layers + [HIDDEN]
        self.outs = [HIDDEN] * (2 + 2 * layers) + [outputs]
        self.layers = layers
        self.p = torch.tensor(np.asarray(params, np.float32), requires_grad=True)

    def _mlps(self):
        off = 0
        out = []
        for k, o in zip(self.kin, self.outs):
            w1 = self.p[off:off + k * HIDDEN].view(k, HIDDEN)
            off += k * HIDDEN
            b1 = self.p[off:off + HIDDEN]
            off += HIDDEN
            w2 = self.p[off:off + HIDDEN * o].view(HIDDEN, o)
            off += HIDDEN * o
            b2 = self.p[off:off + o]
            off += o
            out.append((w1, b1, w2, b2))
        return out

    @staticmethod
    def _mlp(x, m, bf16):
        w1, b1, w2, b2 = m
        z = _r(x, bf16) @ _r(w1, bf16) + b1
        return _r(torch.relu(z), bf16) @ _r(w2, bf16) + b2

    def forward(self, xn, xe, src, dst, bf16=True):
        m = self._mlps()
        src = torch.as_tensor(src, dtype=torch.long)
        dst = torch.as_tensor(dst, dtype=torch.long)
        h = self._mlp(torch.as_tensor(xn, dtype=torch.float32), m[0], bf16)
        e = self._mlp(torch.as_tensor(xe, dtype=torch.float32), m[1], bf16)
        for l in range(self.layers):
            e = e + self._mlp(torch.cat([e, h[src], h[dst]], 1), m[2 + 2 * l], bf16)
            agg = torch.zeros_like(h).index_add_(0, dst, e)
            h = h + self._mlp(torch.cat([h, agg], 1), m[3 + 2 * l], bf16)
        return self._mlp(h, m[-1], bf16)

    def loss_and_grad(self, xn, xe, src, dst, target, bf16=True):
        self.p.grad = None
        y = self.forward(xn, xe, src, dst, bf16)
        loss = ((y - torch.as_tensor(target, dtype=torch.float32)) ** 2).mean()
        loss.backward()
        return float(loss.detach()), self.p.grad.detach().numpy().copy()
