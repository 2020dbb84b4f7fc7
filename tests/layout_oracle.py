"""The device layout's rules restated in numpy: test infrastructure for
tests/test_gpu_layout.py, which holds the arrays layout.cu builds on the GPU
to these bit for bit.

Rules (the library's own data layout, not the reference's):
  cells     identity, or reverse Cuthill-McKee from the internal faces
            (renumber = 1);
  faces     internal faces by (new owner // 4096, upwind signature, new
            owner % 4096, new neighbour, caller face), then boundary faces
            by new owner (stable);
  stencil   slot k of new cell i holds the caller's k-th stencil entry of
            the cell, weights LHS^-1 . RHS_e from the least-squares export;
  gather    per new cell, (face << 1) | side over its faces, ascending.
"""

from collections import deque

import numpy as np

WINDOW = 4096
E = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1], [1, 1, -1], [1, -1, 1], [-1, 1, 1]],
             np.float64)


def rcm_order(C, Fi, owner, nb):
    """order[new] = caller cell: the start cells by ascending degree (stable),
    breadth-first with neighbours by ascending degree (stable), reversed."""
    owner, nb = owner[:Fi], nb[:Fi]
    deg = np.bincount(owner, minlength=C) + np.bincount(nb, minlength=C)
    adj = [[] for _ in range(C)]
    for o, n in zip(owner.tolist(), nb.tolist()):
        adj[o].append(n)
        adj[n].append(o)
    seen = np.zeros(C, bool)
    order = []
    for s in sorted(range(C), key=lambda i: deg[i]):
        if seen[s]:
            continue
        seen[s] = True
        q = deque([s])
        while q:
            v = q.popleft()
            order.append(v)
            for w in sorted(adj[v], key=lambda i: deg[i]):
                if not seen[w]:
                    seen[w] = True
                    q.append(w)
    return np.array(order[::-1], np.int32)


def signature(normal, dt):
    """Base-3 branch code over the 7 lattice pairs (1: e.n > 0.001 dt,
    2: e.n < -0.001 dt), the sum e.n taken left to right as the kernels do."""
    d1 = 0.001 * dt
    sig = np.zeros(len(dt), np.int64)
    p3 = 1
    for e in E:
        s = e[0] * normal[:, 0] + e[1] * normal[:, 1] + e[2] * normal[:, 2]
        sig += p3 * np.where(s > d1, 1, np.where(s < -d1, 2, 0))
        p3 *= 3
    return sig


def expected_layout(ma, cell_order, lhs_inv, rhs):
    """The layout of mesh `ma` for the cell order `cell_order` and the
    least-squares matrices (lhs_inv [C,3,3], rhs [nnz,3], caller numbering)."""
    C, F, Fi = ma.n_cells, ma.n_faces, ma.n_internal
    owner = np.asarray(ma.owner, np.int64)
    nb = np.asarray(ma.neighbour, np.int64)
    cell_new = np.empty(C, np.int64)
    cell_new[cell_order] = np.arange(C)
    f_int = np.arange(Fi)
    o = cell_new[owner[:Fi]]
    n = cell_new[nb[:Fi]]
    normal = np.asarray(ma.face_normal, np.float64).reshape(-1, 3)
    sig = signature(normal[:Fi], np.asarray(ma.streaming_dt, np.float64)[:Fi])
    internal = f_int[np.lexsort((f_int, n, o % WINDOW, sig, o // WINDOW))]
    f_bnd = np.arange(Fi, F)
    boundary = f_bnd[np.argsort(cell_new[owner[Fi:]], kind="stable")]
    face_order = np.concatenate([internal, boundary]).astype(np.int32)
    bc_new = np.empty(F - Fi, np.int64)
    bc_new[boundary - Fi] = np.arange(F - Fi)

    off = np.asarray(ma.stencil_offsets, np.int64)
    cells = np.asarray(ma.stencil_cells, np.int64)
    counts = np.diff(off)
    K = int(counts.max())
    owner_of_e = np.repeat(np.arange(C), counts)
    slot = np.arange(off[-1]) - off[owner_of_e]
    tgt = slot * C + cell_new[owner_of_e]
    nbr_new = np.where(cells < C, cell_new[np.minimum(cells, C - 1)],
                       C + bc_new[np.maximum(cells - C, 0)])
    st_nbr = np.full(K * C, -1, np.int32)
    st_nbr[tgt] = nbr_new
    L = lhs_inv[owner_of_e]
    r = rhs
    st_w = np.zeros((3, K * C))
    for c in range(3):
        st_w[c, tgt] = L[:, c, 0] * r[:, 0] + L[:, c, 1] * r[:, 1] + L[:, c, 2] * r[:, 2]

    k = np.arange(F)
    own_new = cell_new[owner[face_order]]
    cell = np.concatenate([own_new, cell_new[nb[face_order[:Fi]]]])
    val = np.concatenate([k << 1, (k[:Fi] << 1) | 1])
    idx = np.lexsort((val, cell))
    cell, val = cell[idx], val[idx]
    counts2 = np.bincount(cell, minlength=C)
    K2 = int(counts2.max())
    start = np.concatenate([[0], np.cumsum(counts2)[:-1]])
    slot2 = np.arange(len(cell)) - start[cell]
    gather = np.full(K2 * C, -1, np.int32)
    gather[slot2 * C + cell] = val
    return dict(face_order=face_order, stencil_nbr=st_nbr.reshape(K, C),
                stencil_w=st_w.reshape(3, K, C), gather=gather.reshape(K2, C))
