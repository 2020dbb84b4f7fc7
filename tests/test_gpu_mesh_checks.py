"""plfbs_create checks the caller's mesh on the device when one is present
(the arrays are copied there first) and on the host threads otherwise. Both
report the first failing index of the same checks with the same message: each
corrupt mesh below is created on device 0 and on a device index that does not
exist (host checks, which come before the missing device is reported), and
the errors must be identical. A mesh that passes gives the same solver
either way (covered by every other GPU test)."""

import copy

import numpy as np
import pytest

import golden_cases
from plfbs import capi, cases

pytestmark = pytest.mark.gpu


def _cavity():
    d = golden_cases.build("cavity")
    rt, vt, val = cases.bc_arrays(d["ma"], d["case"])
    return d["ma"], rt, vt, val


def _error(ma, rt, vt, val, device):
    cfg = dict(visc=0.006, dt=0.1, max_velocity=0.1, lengths=(6, 5, 4))
    with pytest.raises(capi.PlfbsError) as e:
        capi.Solver(ma, rt, vt, val, cfg, device=device)
    return e.value.code, str(e.value)


def _set(ma, name, index, value):
    bad = copy.deepcopy(ma)
    arr = np.array(getattr(bad, name), copy=True)
    arr.reshape(-1)[index] = value
    setattr(bad, name, arr)
    return bad


CORRUPT = [
    ("owner", 5, -1),                       # face owner out of range
    ("owner", 40, 10 ** 6),
    ("neighbour", 3, "ghost"),              # internal face pointing at a ghost
    ("neighbour", "boundary", 0),           # boundary face not n_cells + face - n_internal
    ("owner", "boundary", -1),              # a boundary face's owner out of range: the host's
    ("owner", "boundary", 10 ** 6),         # boundary order meanwhile guards its indexing
    ("face_area", 17, 0.0),                 # area not positive
    ("face_area", 2, np.nan),
    ("streaming_dt", 9, -0.5),
    ("face_normal", 3 * 11 + 1, np.inf),
    ("cell_volume", 2, -1.0),
    ("cell_volume", 7, np.nan),
    ("stencil_offsets", 4, "decrease"),     # stencil offsets decrease
    ("stencil_cells", 0, "not_neighbour"),  # not a face neighbour of cell 0
    ("stencil_cells", 9, -3),               # out of range
    ("stencil_faces", 12, 10 ** 7),
]


@pytest.mark.parametrize("name,index,value", CORRUPT)
def test_device_checks_report_as_the_host(plfbs_lib, name, index, value):
    ma, rt, vt, val = _cavity()
    if value == "ghost":
        value = ma.n_cells + 7
    if index == "boundary":
        index = ma.n_internal + 4
    if value == "decrease":
        value = int(ma.stencil_offsets[index - 1]) - 1
    if value == "not_neighbour":
        value = int(ma.stencil_cells[7])
    bad = _set(ma, name, index, value)
    dev = _error(bad, rt, vt, val, 0)
    host = _error(bad, rt, vt, val, 99)
    assert dev == host
    assert dev[0] == capi.ERR_MESH


def test_two_faults_report_the_first(plfbs_lib):
    """Several failing faces and cells: the smallest index of the first
    check in the host's order is the one reported."""
    ma, rt, vt, val = _cavity()
    bad = _set(ma, "face_area", 30, -1.0)
    bad = _set(bad, "face_area", 12, 0.0)
    bad = _set(bad, "owner", 50, -4)
    bad = _set(bad, "cell_volume", 1, 0.0)
    dev = _error(bad, rt, vt, val, 0)
    assert dev == _error(bad, rt, vt, val, 99)
    assert "(index 12," in dev[1]
