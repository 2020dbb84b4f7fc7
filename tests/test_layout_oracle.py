"""Self-consistency of the numpy restatement of the device layout
(tests/layout_oracle.py), which tests/test_gpu_layout.py holds the GPU-built
layout to: orders are permutations, the face order keeps its grouping keys
sorted, every face reaches its cells through the gather, stencils are valid."""

import numpy as np
import pytest

import golden_cases
import layout_oracle
from plfbs import capi, cases


def _meshes():
    yield "cavity", golden_cases.build("cavity")["ma"]
    yield "box", cases.mesh_arrays(cases.uniform_box(20, 9, 7), 0.01, 1.0, 0.0)
    yield "tets", cases.mesh_arrays(cases.jittered_tet_box(4, jitter=0.1, seed=2), 0.01, 1.0, 0.0)


@pytest.mark.parametrize("name,ma", list(_meshes()), ids=lambda v: v if isinstance(v, str) else "")
def test_layout_oracle_is_consistent(name, ma):
    C, F, Fi = ma.n_cells, ma.n_faces, ma.n_internal
    owner, nb = np.asarray(ma.owner), np.asarray(ma.neighbour)
    order = layout_oracle.rcm_order(C, Fi, owner, nb)
    assert sorted(order.tolist()) == list(range(C))
    lhs, rhs = capi.ls_weights(ma, capi.GRAD_LS)
    for cell_order in (np.arange(C, dtype=np.int32), order):
        L = layout_oracle.expected_layout(ma, cell_order, lhs, rhs)
        fo = L["face_order"]
        assert sorted(fo.tolist()) == list(range(F))
        assert (fo[:Fi] < Fi).all() and (fo[Fi:] >= Fi).all()
        cell_new = np.empty(C, np.int64)
        cell_new[cell_order] = np.arange(C)
        o = cell_new[owner[fo[:Fi]]]
        sig = layout_oracle.signature(np.asarray(ma.face_normal)[fo[:Fi]],
                                      np.asarray(ma.streaming_dt)[fo[:Fi]])
        key = (o // layout_oracle.WINDOW) * 3 ** 7 + sig
        assert (np.diff(key) >= 0).all()  # window, then signature, non-decreasing
        ob = cell_new[owner[fo[Fi:]]]
        assert (np.diff(ob) >= 0).all()  # boundary faces by new owner
        g = L["gather"]
        vals = g[g >= 0]
        faces, sides = vals >> 1, vals & 1
        assert np.bincount(faces, minlength=F)[:Fi].tolist() == [2] * Fi
        assert np.bincount(faces, minlength=F)[Fi:].tolist() == [1] * (F - Fi)
        assert (sides[faces >= Fi] == 0).all()
        st = L["stencil_nbr"]
        assert ((st >= -1) & (st < C + (F - Fi))).all()
        filled = st >= 0
        assert (filled[:-1] | ~filled[1:]).all()  # empty slots only at the end of a cell's list


@pytest.mark.parametrize("name,ma", list(_meshes()), ids=lambda v: v if isinstance(v, str) else "")
def test_library_cell_order_matches_the_oracle(plfbs_lib, name, ma):
    """plfbs_cell_order (the order plfbs_create renumbers with) against the numpy
    restatement of RCM; renumber 0 is the identity."""
    want = layout_oracle.rcm_order(ma.n_cells, ma.n_internal, np.asarray(ma.owner),
                                   np.asarray(ma.neighbour))
    np.testing.assert_array_equal(capi.cell_order(ma, 1), want)
    np.testing.assert_array_equal(capi.cell_order(ma, 0), np.arange(ma.n_cells))
    np.testing.assert_array_equal(capi.cell_order(ma, 2), want)  # the device order's target
    with pytest.raises(capi.PlfbsError):
        capi.cell_order(ma, 3)
