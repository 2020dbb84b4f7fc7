"""The C-ABI library on CPU: it loads, exports every symbol include/plfbs.h
declares, computes the least-squares weights on the host exactly as the
reference does, and rejects bad input before touching a GPU."""

import ctypes as C
import os
import re

import numpy as np
import pytest

import golden_cases
from conftest import REPO, load_golden
from plfbs import capi, cases, gnn


def _declared():
    src = "".join(open(os.path.join(REPO, "include", f)).read()
                  for f in sorted(os.listdir(os.path.join(REPO, "include"))) if f.endswith(".h"))
    return sorted(set(re.findall(r"\b(plfbs_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol(plfbs_lib):
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(plfbs_lib, n), n
    assert set(names) == set(capi.EXPORTS) | set(gnn.EXPORTS)
    assert plfbs_lib.plfbs_version().startswith(b"plfbs-b200")


@pytest.mark.parametrize("name", golden_cases.NAMES)
def test_host_ls_weights_bit_exact(plfbs_lib, name):
    d = golden_cases.build(name)
    g = load_golden(name)
    mode = golden_cases.oracle_cfg(d)["gradient_mode"]
    lhs, rhs = capi.ls_weights(d["ma"], mode)
    np.testing.assert_array_equal(lhs, g["lhs_inv"])
    np.testing.assert_array_equal(rhs.reshape(-1, 6, 3), g["rhs_w"])


def _create(ma, rt, vt, val, **over):
    cfg = dict(visc=0.006, dt=0.1, max_velocity=0.1, lengths=(6, 5, 4))
    cfg.update(over)
    return capi.Solver(ma, rt, vt, val, cfg)


def _cavity():
    d = golden_cases.build("cavity")
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    return d["ma"], rt, vt, val


def test_rejects_undefined_boundary_types(plfbs_lib):
    ma, rt, vt, val = _cavity()
    vt = vt.copy()
    vt[5] = 3  # periodic: CPU-only in the reference (LBFS.cu:1262-1294 has 1, 2, 9)
    with pytest.raises(capi.PlfbsError) as e:
        _create(ma, rt, vt, val)
    assert e.value.code == capi.ERR_BC
    rt = rt.copy()
    rt[0] = 7
    with pytest.raises(capi.PlfbsError) as e:
        _create(ma, rt, vt * 0 + 1, val)
    assert e.value.code == capi.ERR_BC


def test_rejects_corrupt_mesh(plfbs_lib):
    ma, rt, vt, val = _cavity()
    import copy
    bad = copy.deepcopy(ma)
    bad.neighbour = bad.neighbour.copy()
    bad.neighbour[3] = bad.n_cells + 7  # internal face pointing at a ghost
    with pytest.raises(capi.PlfbsError) as e:
        _create(bad, rt, vt, val)
    assert e.value.code == capi.ERR_MESH
    bad = copy.deepcopy(ma)
    bad.stencil_cells = bad.stencil_cells.copy()
    bad.stencil_cells[0] = bad.stencil_cells[7]  # not a face neighbour of cell 0
    with pytest.raises(capi.PlfbsError) as e:
        _create(bad, rt, vt, val)
    assert e.value.code == capi.ERR_MESH
    bad = copy.deepcopy(ma)
    bad.cell_volume = bad.cell_volume.copy()
    bad.cell_volume[2] = -1.0
    with pytest.raises(capi.PlfbsError) as e:
        _create(bad, rt, vt, val)
    assert e.value.code == capi.ERR_MESH


def test_rejects_bad_config(plfbs_lib):
    ma, rt, vt, val = _cavity()
    with pytest.raises(capi.PlfbsError) as e:
        _create(ma, rt, vt, val, dt=0.0)
    assert e.value.code == capi.ERR_ARG


def test_rejects_unknown_renumber(plfbs_lib):
    ma, rt, vt, val = _cavity()
    with pytest.raises(capi.PlfbsError) as e:
        _create(ma, rt, vt, val, renumber=3)
    assert e.value.code == capi.ERR_ARG and "renumber" in str(e.value)


def test_context_free_errors_are_per_thread(plfbs_lib):
    """plfbs_last_error(NULL) keeps each thread's own last failure: two threads
    fail differently, each waits for the other's failure, then reads."""
    import threading
    L = capi.lib()
    gate = threading.Barrier(2)
    seen = {}

    def fail(name, call):
        assert call() != 0
        gate.wait(timeout=30)
        seen[name] = L.plfbs_last_error(None)

    a = threading.Thread(target=fail, args=("pool", lambda: L.plfbs_release_cached(-1)))
    b = threading.Thread(target=fail, args=("null", lambda: L.plfbs_cell_order(None, 0, None)))
    for t in (a, b):
        t.start()
    for t in (a, b):
        t.join(timeout=60)
    assert b"device index" in seen["pool"]
    assert seen["null"] == b"null argument"


def test_c_program_links_the_library(plfbs_lib, tmp_path):
    """The public headers compile as strict C99 and a C program calls the
    library's host-only entry points (tests/c_abi_check.c)."""
    import subprocess
    libdir = os.path.dirname(capi.LIB_PATH)
    exe = str(tmp_path / "c_abi_check")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "c_abi_check.c"), "-o", exe,
                    "-L" + libdir, "-lplfbs", "-Wl,-rpath," + libdir], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.startswith("plfbs")


def test_null_context_calls_fail_cleanly(plfbs_lib):
    assert plfbs_lib.plfbs_run_stages(None, 1) == capi.ERR_ARG
    assert plfbs_lib.plfbs_set_debug(None, 1) == capi.ERR_ARG
    assert plfbs_lib.plfbs_set_timeout(None, 1.0) == capi.ERR_ARG
    assert plfbs_lib.plfbs_wait(None, 1.0) == capi.ERR_ARG
    plfbs_lib.plfbs_destroy(None)


def _tets(n=4, seed=3):
    pm = cases.jittered_tet_box(n, jitter=0.2, seed=seed,
                                patch_types=["wall", "wall", "wall", "lid", "wall", "wall"])
    c = cases.Case(mesh_dir="", X=n, Y=n, Z=n, dt=0.02, mach=0.1, reynolds=100, ref_length=n,
                   bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet", "neumann"),
                        cases.BC("lid", 1, 1, 0, 0, "dirichlet", "neumann")])
    return cases.mesh_arrays(pm, c.visc, c.gamma, c.fneq_min), c


def test_release_cached_checks_device_index(plfbs_lib):
    L = capi.lib()
    assert L.plfbs_release_cached(-1) == capi.ERR_ARG
    assert b"device index" in L.plfbs_last_error(None)
    assert L.plfbs_release_cached(63) == 0  # no pool was made for it: nothing to do


def test_tet_mesh_is_valid():
    """Jittered hexes split into 6 tets: conforming, positive, closed cells."""
    ma, c = _tets()
    V = ma.cell_volume[: ma.n_cells]
    assert V.min() > 0 and abs(V.sum() - 64.0) < 1e-9
    assert set(np.diff(ma.stencil_offsets)) == {4}
    nA = ma.face_normal * ma.face_area[:, None]
    acc = np.zeros((ma.n_cells, 3))
    np.add.at(acc, ma.owner, nA)
    np.add.at(acc, ma.neighbour[: ma.n_internal], -nA[: ma.n_internal])
    assert np.abs(acc).max() < 1e-12


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_exact_inverse_option(plfbs_lib, mode):
    """PLFBS_GRAD_EXACT_INVERSE: the true inverse of the LS matrix; without it
    the reference's determinant (which flips sign on some tets)."""
    import oracle

    ma, _ = _tets()
    lhs_x, rhs_x = capi.ls_weights(ma, mode | capi.GRAD_EXACT_INVERSE)
    lo, ro = oracle.ls_weights(ma, mode | 0x100)
    np.testing.assert_array_equal(lhs_x, lo)
    np.testing.assert_array_equal(rhs_x, ro)
    lhs_r, _ = capi.ls_weights(ma, mode)
    lr, _ = oracle.ls_weights(ma, mode)
    np.testing.assert_array_equal(lhs_r, lr)
    # the exact inverse inverts the LHS rebuilt from the same formula
    C = ma.n_cells
    for i in range(0, C, 37):
        L = np.zeros((3, 3))
        e0, e1 = ma.stencil_offsets[i], ma.stencil_offsets[i + 1]
        for e in range(e0, e1):
            f, i1 = ma.stencil_faces[e], ma.stencil_cells[e]
            d = ma.cell_centroid[i1] - ma.cell_centroid[i]
            ln = (ma.face_centroid[f] - ma.cell_centroid[i]) @ ma.face_normal[f]
            w = (2 * ln / (d @ ma.face_normal[f])) ** 2 * ma.face_area[f] / np.sqrt(d @ d)
            L += w * np.outer(d, d)
        if mode == 0:
            np.testing.assert_allclose(lhs_x[i] @ L, np.eye(3), atol=1e-12)


def test_polymesh_geometry_rejects_bad_indices(plfbs_lib):
    """The polyMesh's indices are checked on the host before any device work."""
    import copy
    pm = golden_cases.build("cavity")["pm"]
    bad = copy.deepcopy(pm)
    bad.faces = bad.faces.copy()
    bad.faces[5, 2] = bad.points.shape[0]  # vertex out of range
    with pytest.raises(capi.PlfbsError) as e:
        capi.polymesh_geometry(bad, 0.01, 1.0, 0.0)
    assert e.value.code == capi.ERR_MESH and "vertex" in str(e.value)
    bad = copy.deepcopy(pm)
    bad.nverts = bad.nverts.copy()
    bad.nverts[3] = 2  # a face needs three vertices
    with pytest.raises(capi.PlfbsError) as e:
        capi.polymesh_geometry(bad, 0.01, 1.0, 0.0)
    assert e.value.code == capi.ERR_MESH
    bad = copy.deepcopy(pm)
    bad.neighbour = bad.neighbour.copy()
    bad.neighbour[0] = bad.owner[0]
    with pytest.raises(capi.PlfbsError) as e:
        capi.polymesh_geometry(bad, 0.01, 1.0, 0.0)
    assert e.value.code == capi.ERR_MESH
    with pytest.raises(capi.PlfbsError) as e:
        capi.polymesh_geometry(pm, 0.01, 0.0, 0.0)
    assert e.value.code == capi.ERR_ARG


def test_flavour_boundary_tables(plfbs_lib):
    """Each flavour takes its own reference solver's boundary types; checked
    on the host, so a case that passes reaches the device check."""
    d = golden_cases.build_cpu("cpu_channel")
    ma = d["ma"]
    rt, vt, val = cases.bc_arrays(ma, d["case"])
    assert set(vt) == {1, 2, 6, 8} and set(rt) == {1, 2, 7}
    cfg = dict(golden_cases.oracle_cfg(d))
    with pytest.raises(capi.PlfbsError) as e:  # GPU kernels: types 1, 2, 9 only
        capi.Solver(ma, rt, vt, val, cfg)
    assert e.value.code == capi.ERR_BC
    cpu = dict(cfg, flavour=capi.FLAVOUR_CPU_SOLVER)
    try:  # valid: fails only for want of a device
        capi.Solver(ma, rt, vt, val, cpu).close()
    except capi.PlfbsError as e:
        assert e.code == capi.ERR_NO_DEVICE
    bad = vt.copy()
    bad[0] = 9  # parabolic: GPU path only
    with pytest.raises(capi.PlfbsError) as e:
        capi.Solver(ma, rt, bad, val, cpu)
    assert e.value.code == capi.ERR_BC
    bad = rt.copy()
    bad[0] = 8  # the reference never writes this ghost's density gradient
    with pytest.raises(capi.PlfbsError) as e:
        capi.Solver(ma, bad, vt, val, cpu)
    assert e.value.code == capi.ERR_BC
    with pytest.raises(capi.PlfbsError) as e:
        capi.Solver(ma, rt, vt, val, dict(cpu, precision=capi.FP32_DEVIATION))
    assert e.value.code == capi.ERR_ARG
    nodes = np.zeros((2, 3)) + 3.0
    with pytest.raises(capi.PlfbsError) as e:
        capi.Solver(ma, rt, vt, val, cpu, ibm=dict(node_ref=nodes, object_nodes=2))
    assert e.value.code == capi.ERR_ARG
    with pytest.raises(capi.PlfbsError) as e:
        capi.Solver(ma, rt, vt, val, dict(cfg, flavour=2))
    assert e.value.code == capi.ERR_ARG


@pytest.mark.parametrize("name", golden_cases.CPU_NAMES)
def test_cpu_solver_fixtures(name):
    d = golden_cases.build_cpu(name)
    g = load_golden(name)
    np.testing.assert_array_equal(d["state0"], g["state_init"])
    assert g["final_state"].shape == (d["ma"].total_cells, 4)
    assert np.isfinite(g["final_state"]).all()
