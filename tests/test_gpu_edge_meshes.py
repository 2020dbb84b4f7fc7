"""Edge cases of the device-built geometry and layout: a single cell (no
internal face), one-cell-thick strips, a handful of tetrahedra. The geometry
from the polyMesh must equal the numpy restatement bit for bit, and a few
steps must match the C oracle (GPU-kernel semantics) to 1e-10."""

import numpy as np
import pytest

import oracle
from conftest import rel_l2
from plfbs import capi, cases

pytestmark = pytest.mark.gpu

KEYS = ("owner", "neighbour", "face_area", "face_normal", "face_centroid", "streaming_dt",
        "cell_volume", "cell_centroid", "stencil_offsets", "stencil_cells", "stencil_faces")


def _mesh(kind):
    if kind == "cell":
        return cases.uniform_box(1, 1, 1, patch_types=["wall", "wall", "wall", "lid", "wall",
                                                       "wall"]), (1, 1, 1)
    if kind == "strip":
        return cases.uniform_box(2, 1, 1, patch_types=["wall", "wall", "wall", "lid", "wall",
                                                       "wall"]), (2, 1, 1)
    if kind == "slab":
        return cases.uniform_box(3, 2, 1, patch_types=["wall", "wall", "wall", "lid", "wall",
                                                       "wall"]), (3, 2, 1)
    return cases.jittered_tet_box(1, jitter=0.0, seed=1,
                                  patch_types=["wall", "wall", "wall", "lid", "wall",
                                               "wall"]), (1, 1, 1)


@pytest.mark.parametrize("kind", ["cell", "strip", "slab", "tets"])
def test_tiny_meshes(plfbs_lib, kind):
    pm, (X, Y, Z) = _mesh(kind)
    c = cases.Case(mesh_dir="", X=X, Y=Y, Z=Z, dt=0.05, mach=0.1, reynolds=10.0, ref_length=1.0,
                   tolerance=0.0,
                   bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann"),
                        cases.BC("lid", 1, 1, 0, 0, "dirichlet", "neumann")])
    ma = cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min)
    g = capi.polymesh_geometry(pm, c.visc, c.gamma, c.fneq_min)
    for key in KEYS:
        np.testing.assert_array_equal(getattr(g, key), getattr(ma, key), err_msg=key)
    rt, vt, val = cases.bc_arrays(ma, c)
    T = ma.total_cells
    rng = np.random.default_rng(5)
    s0 = np.zeros((T, 4))
    s0[:, :3] = 0.01 * rng.standard_normal((T, 3))
    s0[:, 3] = 1.0 + 0.001 * rng.standard_normal(T)
    cfg = dict(visc=c.visc, gamma=1.0, dt=c.dt, domain_dt=0.5, pressure_gradient=0.0,
               channel_height=c.Y, max_velocity=c.mach, ref_rho=1.0, tolerance=0.0,
               origin=(0, 0, 0), lengths=(c.X, c.Y, c.Z), gradient_mode=capi.GRAD_LS)
    o = oracle.OracleRun(ma, rt, vt, val, cfg, s0)
    o.run_steps(5)
    for renumber in (0, 1, 2):
        s = capi.Solver(ma, rt, vt, val, dict(cfg, renumber=renumber))
        s.set_state(s0)
        s.run(5)
        st = s.get_state()
        for k in range(4):
            assert rel_l2(st[: ma.n_cells, k], o.state[: ma.n_cells, k]) < 1e-10, (renumber, k)
        assert s.wall_forces([]) == (0.0, 0.0)
        walls = [i for i, t in enumerate(ma.bc_types) if t == "wall"]
        cd, cl = s.wall_forces(walls)
        assert np.isfinite(cd) and np.isfinite(cl)
        s.close()
