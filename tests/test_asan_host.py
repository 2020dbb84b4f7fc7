"""The library's host-side setup (csrc/setup.cpp) under AddressSanitizer
(tests/asan_setup_check.cpp): the layout's checks, the cell orders, the
boundary records and the least-squares export on valid meshes (one large
enough for the multi-threaded checks, one with enough boundary faces for the
multi-threaded key sort) and on corrupt ones of every kind the checks reject.
The path plfbs_create takes with a device (the host's share of the layout on
unchecked arrays, then the checks' results) must give the same status,
message and boundary records as the checks-first path. The arrays are exactly
the sizes the C ABI promises, so any access beyond what a caller hands over
ends the run with a report."""

import copy
import os
import shutil
import subprocess

import numpy as np
import pytest

import golden_cases
from conftest import REPO
from plfbs import capi, cases

CSRC = os.path.join(REPO, "3d-plfbs-gpu_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    exe = str(tmp_path_factory.mktemp("asan") / "asan_setup_check")
    r = subprocess.run([gxx, "-std=c++17", "-O1", "-g", "-fsanitize=address",
                        "-fno-omit-frame-pointer", "-pthread", "-I", os.path.join(REPO, "include"),
                        "-I", CSRC, "-I", "/usr/local/cuda/include",
                        os.path.join(REPO, "tests", "asan_setup_check.cpp"),
                        os.path.join(CSRC, "setup.cpp"), "-o", exe], capture_output=True, text=True)
    if r.returncode != 0 and ("-lasan" in r.stderr or "libasan" in r.stderr):
        pytest.skip("this g++ has no AddressSanitizer runtime")
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


def _write(d, ma, rt, vt, val):
    os.makedirs(d)
    a = lambda x, t: np.ascontiguousarray(x, t).tofile  # noqa: E731
    nnz = len(ma.stencil_cells)
    with open(os.path.join(d, "meta.txt"), "w") as f:
        f.write("%d %d %d %d\n" % (ma.n_cells, ma.n_faces, ma.n_internal, nnz))
    for name, x, t in (("owner", ma.owner, np.int32), ("neighbour", ma.neighbour, np.int32),
                       ("face_area", ma.face_area, np.float64),
                       ("face_normal", ma.face_normal, np.float64),
                       ("face_centroid", ma.face_centroid, np.float64),
                       ("streaming_dt", ma.streaming_dt, np.float64),
                       ("cell_volume", ma.cell_volume, np.float64),
                       ("cell_centroid", ma.cell_centroid, np.float64),
                       ("stencil_offsets", ma.stencil_offsets, np.int32),
                       ("stencil_cells", ma.stencil_cells, np.int32),
                       ("stencil_faces", ma.stencil_faces, np.int32),
                       ("rho_type", rt, np.int32), ("vel_type", vt, np.int32),
                       ("bc_value", val, np.float64)):
        a(x, t)(os.path.join(d, name))


def _corrupt(ma, rt, vt, val, kind):
    ma = copy.deepcopy(ma)
    rt, vt, val = rt.copy(), vt.copy(), val.copy()
    C, Fi = ma.n_cells, ma.n_internal
    T = ma.total_cells

    def arr(name):
        x = np.array(getattr(ma, name), copy=True)
        setattr(ma, name, x)
        return x

    if kind == "owner":
        arr("owner")[3] = C + 7
    elif kind == "neighbour":
        arr("neighbour")[2] = C + 1
    elif kind == "ghost":
        arr("neighbour")[Fi] = 0
    elif kind == "stencil_cell":
        arr("stencil_cells")[5] = T + 100
    elif kind == "stencil_face":
        arr("stencil_faces")[5] = ma.n_faces + 3
    elif kind == "stencil_face_neg":
        arr("stencil_faces")[5] = -1
    elif kind == "stencil_not_neighbour":
        arr("stencil_cells")[0] = ma.stencil_cells[7]
    elif kind == "offsets":
        off = arr("stencil_offsets")
        off[4] = off[5] + 1
    elif kind == "volume":
        arr("cell_volume")[2] = -1.0
    elif kind == "area":
        arr("face_area")[0] = np.nan
    elif kind == "bc_type":
        rt[0] = 5
    elif kind == "owner_boundary_low":  # the deferred boundary order guards these
        arr("owner")[Fi + 3] = -5
    elif kind == "owner_boundary_high":
        arr("owner")[Fi + 3] = C + 1000
    return ma, rt, vt, val


KINDS = ("owner", "neighbour", "ghost", "stencil_cell", "stencil_face", "stencil_face_neg",
         "stencil_not_neighbour", "offsets", "volume", "area")


def test_setup_is_memory_clean_on_valid_and_corrupt_meshes(checker, tmp_path):
    d = golden_cases.build("cavity")
    ma0 = d["ma"]
    rt0, vt0, val0 = cases.bc_arrays(ma0, d["case"])
    runs = {"cavity": (ma0, rt0, vt0, val0)}
    box = cases.mesh_arrays(cases.uniform_box(40, 30, 30), 0.01, 1.0, 0.0)
    assert box.n_cells > 32768  # the checks run on several host threads
    c = cases.Case(mesh_dir="", X=40, Y=30, Z=30, bcs=[cases.BC("wall", 1, 0, 0, 0, "dirichlet",
                                                                "neumann")])
    runs["box"] = (box, *cases.bc_arrays(box, c))
    tets = cases.mesh_arrays(cases.jittered_tet_box(4, jitter=0.2, seed=3), 0.01, 1.0, 0.0)
    runs["tets"] = (tets, *cases.bc_arrays(tets, c))
    slab = cases.mesh_arrays(cases.uniform_box(256, 256, 2), 0.01, 1.0, 0.0)
    assert slab.n_faces - slab.n_internal > 65536  # the boundary keys sort on several threads
    runs["slab"] = (slab, *cases.bc_arrays(slab, c))
    for kind in ("owner_boundary_low", "owner_boundary_high"):
        runs[kind] = _corrupt(ma0, rt0, vt0, val0, kind)
    for kind in KINDS + ("bc_type",):
        runs[kind] = _corrupt(ma0, rt0, vt0, val0, kind)
    dirs = []
    for name, (ma, rt, vt, val) in runs.items():
        dirs.append(str(tmp_path / name))
        _write(dirs[-1], ma, rt, vt, val)
    r = subprocess.run([checker, *dirs], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=0:halt_on_error=1"))
    assert r.returncode == 0, r.stderr[-4000:]
    got = {}
    for line in r.stdout.splitlines():
        name, *kv = line.split()
        got[os.path.basename(name)] = {k: int(v) for k, v in (x.split("=") for x in kv)}
    assert set(got) == set(runs)
    for name in ("cavity", "box", "slab"):  # hexes: every call succeeds
        assert all(v == capi.OK for k, v in got[name].items() if not k.startswith("deferred")), (
            name, got[name])
    assert all(v == capi.OK for k, v in got["tets"].items() if k.startswith("layout"))
    for kind in KINDS + ("owner_boundary_low", "owner_boundary_high"):  # rejected by every call
        assert all(v in (capi.ERR_ARG, capi.ERR_MESH) for k, v in got[kind].items()
                   if not k.startswith("deferred")), (kind, got[kind])
    for name, g in got.items():  # the deferred path: the same status, message and records
        assert all(v == 1 for k, v in g.items() if k.startswith("deferred")), (name, g)
        assert sum(k.startswith("deferred") for k in g) == 4, (name, g)
    bc = got["bc_type"]  # a boundary type neither flavour takes: the layout only
    assert all(bc[k] == capi.ERR_BC for k in bc if k.startswith("layout"))
    assert all(bc[k] == capi.OK for k in bc if k.startswith("ls"))
