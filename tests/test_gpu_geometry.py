"""plfbs_polymesh_geometry (the reference's mesh pre-processing on the GPU)
against the reference's own arrays (golden fixtures, dumped by its
unstructured_mesh from the same polyMesh) and against cases.mesh_arrays on
graded, tetrahedral and larger hex meshes: bit for bit."""

import numpy as np
import pytest

import golden_cases
from conftest import load_golden
from plfbs import capi, cases

pytestmark = pytest.mark.gpu

KEYS = ("owner", "neighbour", "face_area", "face_normal", "face_centroid", "streaming_dt",
        "cell_volume", "cell_centroid", "stencil_offsets", "stencil_cells", "stencil_faces")


@pytest.mark.parametrize("name", golden_cases.NAMES)
def test_geometry_matches_the_reference(plfbs_lib, name):
    g = load_golden(name)
    d = golden_cases.build(name)
    c = d["case"]
    ma = capi.polymesh_geometry(d["pm"], c.visc, c.gamma, c.fneq_min)
    C = ma.n_cells
    for key in KEYS[:8]:
        np.testing.assert_array_equal(getattr(ma, key), g[key], err_msg=key)
    np.testing.assert_array_equal(ma.stencil_cells.reshape(C, 6), g["stencil"])
    for key in KEYS:
        np.testing.assert_array_equal(getattr(ma, key), getattr(d["ma"], key), err_msg=key)


@pytest.mark.parametrize("mesh", ["tets", "graded", "box"])
def test_geometry_matches_mesh_arrays(plfbs_lib, mesh):
    if mesh == "tets":
        pm = cases.jittered_tet_box(10, jitter=0.15, seed=5, patch_types=["wall"] * 6)
    elif mesh == "graded":
        xs = np.cumsum(np.r_[0.0, np.linspace(0.5, 1.5, 24)])
        ys = np.cumsum(np.r_[0.0, np.linspace(1.2, 0.6, 16)])
        zs = np.cumsum(np.r_[0.0, np.full(12, 0.75)])
        pm = cases.hex_box(xs, ys, zs)
    else:
        pm = cases.uniform_box(48, 24, 20)
    visc, gamma, fneq_min = 0.004, 1.0, 0.0
    want = cases.mesh_arrays(pm, visc, gamma, fneq_min)
    got = capi.polymesh_geometry(pm, visc, gamma, fneq_min)
    for key in KEYS:
        np.testing.assert_array_equal(getattr(got, key), getattr(want, key), err_msg=key)
    # with the streaming-dt cap active
    want = cases.mesh_arrays(pm, visc, gamma, 0.05)
    got = capi.polymesh_geometry(pm, visc, gamma, 0.05)
    np.testing.assert_array_equal(got.streaming_dt, want.streaming_dt)
