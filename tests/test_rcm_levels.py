"""The level-by-level Cuthill-McKee steps of the device cell order
(csrc/rcm_levels.hpp, renumber 2) evaluated serially on the host
(tests/rcm_levels_host.cpp) against the sequential order: the library's
host RCM (plfbs_cell_order with renumber 1) on meshes, and the numpy
restatement (layout_oracle.rcm_order) on random graphs with repeated
neighbours, several components and cells without internal faces."""

import ctypes
import os
import subprocess

import numpy as np
import pytest

import golden_cases
import layout_oracle
from conftest import REPO
from plfbs import capi, cases

CSRC = os.path.join(REPO, "3d-plfbs-gpu_b200", "csrc")
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def levels(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("rcm") / "librcm_levels_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC,
                    os.path.join(HERE, "rcm_levels_host.cpp"), "-o", so], check=True)
    lib = ctypes.CDLL(so)
    lib.rcm_by_levels.restype = ctypes.c_int
    i32p = ctypes.POINTER(ctypes.c_int32)

    def run(C, owner, nb):
        owner = np.ascontiguousarray(owner, np.int32)
        nb = np.ascontiguousarray(nb, np.int32)
        out = np.full(C, -1, np.int32)
        bad = lib.rcm_by_levels(C, len(owner), owner.ctypes.data_as(i32p),
                                nb.ctypes.data_as(i32p), out.ctypes.data_as(i32p))
        assert bad == 0
        return out

    return run


def _meshes():
    yield "cavity", golden_cases.build("cavity")["ma"]
    yield "channel", golden_cases.build("channel")["ma"]
    yield "box", cases.mesh_arrays(cases.uniform_box(40, 20, 20), 0.01, 1.0, 0.0)
    yield "tets", cases.mesh_arrays(cases.jittered_tet_box(12, jitter=0.1, seed=3), 0.01, 1.0, 0.0)


@pytest.mark.parametrize("name,ma", list(_meshes()), ids=lambda v: v if isinstance(v, str) else "")
def test_levels_match_the_library_order_on_meshes(plfbs_lib, levels, name, ma):
    Fi = ma.n_internal
    got = levels(ma.n_cells, np.asarray(ma.owner)[:Fi], np.asarray(ma.neighbour)[:Fi])
    np.testing.assert_array_equal(got, capi.cell_order(ma, 1))
    np.testing.assert_array_equal(capi.cell_order(ma, 2), capi.cell_order(ma, 1))


def _random_graph(seed, C, E, isolated, pieces):
    """Internal faces of a random multigraph: `pieces` disjoint blocks of
    cells, repeated pairs, and `isolated` cells touching no internal face."""
    rng = np.random.default_rng(seed)
    cells = rng.permutation(C)
    live, dead = cells[isolated:], cells[:isolated]
    blocks = np.array_split(live, pieces)
    owner, nb = [], []
    for b in blocks:
        if len(b) < 2:
            continue
        for i in range(1, len(b)):  # a spanning path keeps the block connected
            owner.append(b[i - 1])
            nb.append(b[i])
        k = E * len(b) // len(live)
        a = rng.integers(0, len(b), k)
        c = rng.integers(0, len(b), k)
        keep = a != c
        owner.extend(b[a[keep]])
        nb.extend(b[c[keep]])
    owner, nb = np.array(owner, np.int32), np.array(nb, np.int32)
    perm = rng.permutation(len(owner))
    assert not np.isin(dead, owner).any() and not np.isin(dead, nb).any()
    return owner[perm], nb[perm]


@pytest.mark.parametrize("seed,C,E,isolated,pieces", [
    (0, 50, 60, 0, 1), (1, 300, 900, 0, 1), (2, 300, 2000, 5, 1), (3, 1000, 2500, 0, 7),
    (4, 1000, 1200, 40, 3), (5, 2000, 6000, 0, 25), (6, 7, 0, 7, 1), (7, 500, 40, 0, 200)])
def test_levels_match_sequential_rcm_on_random_graphs(levels, seed, C, E, isolated, pieces):
    owner, nb = _random_graph(seed, C, E, isolated, pieces)
    want = layout_oracle.rcm_order(C, len(owner), owner, nb)
    np.testing.assert_array_equal(levels(C, owner, nb), want)
