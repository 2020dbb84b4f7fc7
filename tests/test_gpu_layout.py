"""The layout built on the device (layout.cu) against its rules restated in
numpy (layout_oracle): cell order, face order, stencil neighbours and
weights, and the face-to-cell gather, bit for bit, in both precisions, with
and without RCM renumbering (host order, renumber 1; device order,
renumber 2), on the golden meshes, a hex box of several face windows, a
jittered tetrahedral box and meshes in several disjoint pieces."""

import copy

import numpy as np
import pytest

import golden_cases
import layout_oracle
from plfbs import capi, cases

pytestmark = pytest.mark.gpu


def _check(ma, rt, vt, val, cfg, renumber, precision):
    cfg = dict(cfg, renumber=renumber, precision=precision)
    s = capi.Solver(ma, rt, vt, val, cfg)
    got = s.layout()
    order = got["cell_order"]
    if renumber:
        want = layout_oracle.rcm_order(ma.n_cells, ma.n_internal, np.asarray(ma.owner),
                                       np.asarray(ma.neighbour))
        np.testing.assert_array_equal(order, want)
    else:
        np.testing.assert_array_equal(order, np.arange(ma.n_cells))
    lhs, rhs = capi.ls_weights(ma, cfg.get("gradient_mode", capi.GRAD_LS))
    exp = layout_oracle.expected_layout(ma, order, lhs, rhs)
    np.testing.assert_array_equal(got["face_order"], exp["face_order"])
    np.testing.assert_array_equal(got["stencil_nbr"], exp["stencil_nbr"])
    np.testing.assert_array_equal(got["gather"], exp["gather"])
    w = exp["stencil_w"]
    if precision == capi.FP32_DEVIATION:
        w = w.astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(got["stencil_w"], w)


@pytest.mark.parametrize("precision", [capi.FP64, capi.FP32_DEVIATION])
@pytest.mark.parametrize("renumber", [0, 1, 2])
@pytest.mark.parametrize("name", golden_cases.NAMES)
def test_layout_of_golden_meshes(plfbs_lib, name, renumber, precision):
    d = golden_cases.build(name)
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    _check(d["ma"], rt, vt, val, golden_cases.oracle_cfg(d), renumber, precision)


def _box_case():
    pm = cases.uniform_box(40, 20, 20, patch_types=["inlet", "outlet", "side", "side", "side",
                                                    "side"])
    c = cases.Case(mesh_dir="", X=40, Y=20, Z=20, dt=0.1, mach=0.05, reynolds=100.0,
                   ref_length=8.0,
                   bcs=[cases.BC("inlet", 1, 1, 0, 0, "dirichlet", "neumann"),
                        cases.BC("outlet", 1, 0, 0, 0, "neumann", "dirichlet"),
                        cases.BC("side", 1, 0, 0, 0, "neumann", "neumann")])
    return cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min), c


def _tet_case():
    pm = cases.jittered_tet_box(12, jitter=0.1, seed=3, patch_types=["wall"] * 6)
    c = cases.Case(mesh_dir="", X=12, Y=12, Z=12, dt=0.05, mach=0.05, reynolds=100.0,
                   ref_length=12.0, bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann")])
    return cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min), c


@pytest.mark.parametrize("renumber", [0, 1, 2])
@pytest.mark.parametrize("mesh,mode", [("box", capi.GRAD_LS), ("tets", capi.GRAD_HYBRID),
                                       ("tets", capi.GRAD_LS | capi.GRAD_EXACT_INVERSE)])
def test_layout_of_larger_meshes(plfbs_lib, mesh, mode, renumber):
    ma, c = _box_case() if mesh == "box" else _tet_case()
    assert ma.n_cells > 2 * layout_oracle.WINDOW
    rt, vt, val = cases.bc_arrays(ma, c)
    cfg = dict(visc=c.visc, dt=c.dt, max_velocity=c.mach, channel_height=c.Y,
               lengths=(c.X, c.Y, c.Z), gradient_mode=mode)
    _check(ma, rt, vt, val, cfg, renumber, capi.FP64)


def _join(pms):
    """One polyMesh of disjoint pieces: every piece's internal faces first,
    then every piece's patches, cells and points numbered piece by piece."""
    cell0 = np.cumsum([0] + [pm.n_cells for pm in pms])
    pt0 = np.cumsum([0] + [len(pm.points) for pm in pms])
    V = max(pm.faces.shape[1] for pm in pms)

    def faces(pm, k, rows):
        f = np.full((len(rows), V), -1, np.int32)
        src = pm.faces[rows]
        f[:, :src.shape[1]] = np.where(src >= 0, src + pt0[k], -1)
        return f

    fl, nv, own, nb, patches = [], [], [], [], []
    for k, pm in enumerate(pms):
        rows = np.arange(pm.n_internal)
        fl.append(faces(pm, k, rows))
        nv.append(pm.nverts[rows])
        own.append(pm.owner[rows] + cell0[k])
        nb.append(pm.neighbour + cell0[k])
    start = sum(pm.n_internal for pm in pms)
    for k, pm in enumerate(pms):
        for name, ptype, s0, n in pm.patches:
            rows = np.arange(s0, s0 + n)
            fl.append(faces(pm, k, rows))
            nv.append(pm.nverts[rows])
            own.append(pm.owner[rows] + cell0[k])
            patches.append((name, ptype, start, n))
            start += n
    return cases.PolyMesh(points=np.concatenate([pm.points for pm in pms]).astype(np.float32),
                          faces=np.concatenate(fl), nverts=np.concatenate(nv).astype(np.int32),
                          owner=np.concatenate(own).astype(np.int32),
                          neighbour=np.concatenate(nb).astype(np.int32),
                          n_cells=int(cell0[-1]), patches=patches)


@pytest.mark.parametrize("kind", ["pieces", "many_pieces", "chain"])
def test_device_order_past_its_limits(plfbs_lib, kind):
    """Pieces of different sizes, one of them a single cell (no internal face);
    400 pieces (333 with internal faces) is past the device's component limit
    and a 9,000-cell chain (9,000 levels) past its level budget, where create
    takes the host order (the same order)."""
    if kind == "pieces":
        sizes = [(5, 3, 2), (1, 1, 1), (4, 4, 4)]
    elif kind == "many_pieces":
        sizes = [((k % 3) + 1, 1, (k % 2) + 1) for k in range(400)]
    else:
        sizes = [(9000, 1, 1)]
    pieces = len(sizes)
    pms = [cases.uniform_box(*n, origin=(0.0, 0.0, 10.0 * k)) for k, n in enumerate(sizes)]
    pm = _join(pms)
    c = cases.Case(mesh_dir="", X=5, Y=4, Z=10 * pieces, dt=0.05, mach=0.05, reynolds=100.0,
                   ref_length=4.0, bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann")])
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    rt, vt, val = cases.bc_arrays(ma, c)
    cfg = dict(visc=c.visc, dt=c.dt, max_velocity=c.mach, channel_height=c.Y,
               lengths=(c.X, c.Y, c.Z), gradient_mode=capi.GRAD_LS)
    _check(ma, rt, vt, val, cfg, 2, capi.FP64)


def test_singular_least_squares_matrix_is_reported(plfbs_lib):
    """A cell left with one stencil entry has a rank-1 LS matrix."""
    d = golden_cases.build("cavity")
    ma = copy.deepcopy(d["ma"])
    off = np.asarray(ma.stencil_offsets).copy()
    cells = np.asarray(ma.stencil_cells)
    faces = np.asarray(ma.stencil_faces)
    keep = np.ones(len(cells), bool)
    keep[off[0] + 1:off[1]] = False  # cell 0 keeps its first entry only
    ma.stencil_cells = cells[keep].copy()
    ma.stencil_faces = faces[keep].copy()
    new_off = off.copy()
    new_off[1:] -= off[1] - off[0] - 1
    ma.stencil_offsets = new_off.astype(np.int32)
    rt, vt, val = cases.bc_arrays(ma, d["case"])
    cfg = dict(golden_cases.oracle_cfg(d), gradient_mode=capi.GRAD_LS)
    with pytest.raises(capi.PlfbsError) as e:
        capi.Solver(ma, rt, vt, val, cfg)
    assert e.value.code == capi.ERR_MESH
    assert "singular" in str(e.value)
