"""Synthetic cases for the LBFS time step: OpenFOAM polyMesh + XML writers and
the pre-processed mesh arrays that the reference hands to its GPU solver.

The solver's input boundary is the pre-processed ``unstructured_mesh`` of the
reference (unstructured_mesh.h:15-47): face areas, unit normals and centroids,
cell volumes and centroids (ghost cells included), per-face streaming dt and the
gradient stencil. ``mesh_arrays`` restates how unstructured_mesh.cpp derives
them from a polyMesh so that a case can be built without running the reference:

* points are stored as float32 (unstructured_mesh.h:50, .cpp:300-305) and
  widened to float64;
* each face is fanned from its vertex 0; per triangle the volume contribution
  a . ((b-a) x (c-a)) / 6 goes to the owner and, negated, to the neighbour
  (tet_volume, unstructured_mesh.cpp:577-607, called at :1150-1152);
* area = |(b-a) x (c-a)| / 2, centroid = sum(area * mean(a,b,c)) / area and the
  unit normal is sum((b-a) x (c-a)) normalised (cell_tet_area, :732-766; face
  loop :1154-1182);
* a cell centroid is the area-weighted mean of its face centroids (:1170-1217),
  not the volume centroid;
* a ghost cell (one per boundary face, index n_cells + face - n_internal) sits at
  owner + 2 (face - owner) componentwise scaled by |n| (:1346-1375);
* streaming dt = min(sqrt(A)/2, 3 nu / (gamma fneq_min)) (:979-983);
* the stencil lists, in face order, each cell's face neighbours (:1186-1206).

All accumulations run in the reference's order so the arrays agree bit for bit
with the reference's own (checked against its dumps in the tests).

Synthetic inputs only: structured hex boxes (optionally graded), jittered
hexes split into 6 tetrahedra, Fibonacci-sphere Lagrangian node sets. Every
generator that draws random numbers takes an explicit seed (numpy PCG64).
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

# ----------------------------------------------------------------------------
# polyMesh container
# ----------------------------------------------------------------------------


@dataclass
class PolyMesh:
    """An OpenFOAM polyMesh: float32 points, faces, owner/neighbour and patches.

    ``faces`` is an int32 array [F, maxv] padded with -1, ``nverts`` [F] the
    vertex count of each face. Internal faces come first (owner < neighbour),
    then each patch's faces contiguously, in ``patches`` order.
    """

    points: np.ndarray  # [P, 3] float32
    faces: np.ndarray  # [F, maxv] int32
    nverts: np.ndarray  # [F] int32
    owner: np.ndarray  # [F] int32
    neighbour: np.ndarray  # [F_i] int32
    n_cells: int
    patches: list = field(default_factory=list)  # [(name, type, start, n)]

    @property
    def n_faces(self) -> int:
        return int(self.owner.shape[0])

    @property
    def n_internal(self) -> int:
        return int(self.neighbour.shape[0])

    def bc_types(self) -> list:
        """Per boundary face, the patch *type* string (what the reference keys
        its boundary conditions on, unstructured_mesh.cpp:1912-1987)."""
        out = []
        for _name, ptype, _start, n in self.patches:
            out.extend([ptype] * n)
        return out


def hex_box(xs, ys, zs, patch_types=None) -> PolyMesh:
    """Structured hex mesh on the tensor grid xs x ys x zs (node coordinates).

    Cells are numbered i + j nx + k nx ny (blockMesh order, x fastest), the
    numbering the reference's IBM kernels assume
    (immersed_boundary_method.cu:44-66). Internal faces are in OpenFOAM
    upper-triangular order; patches are x-, x+, y-, y+, z-, z+ with the given
    type strings (default "wall").
    """
    xs = np.asarray(xs, dtype=np.float64)
    ys = np.asarray(ys, dtype=np.float64)
    zs = np.asarray(zs, dtype=np.float64)
    nx, ny, nz = len(xs) - 1, len(ys) - 1, len(zs) - 1
    px, py = nx + 1, ny + 1
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    pts = np.stack([X.transpose(2, 1, 0).ravel(), Y.transpose(2, 1, 0).ravel(),
                    Z.transpose(2, 1, 0).ravel()], axis=1).astype(np.float32)

    def p(i, j, k):
        return i + j * px + k * px * py

    C = nx * ny * nz
    cid = np.arange(C, dtype=np.int64)
    ci, cj, ck = cid % nx, (cid // nx) % ny, cid // (nx * ny)

    # internal faces, per owner in increasing neighbour order: +x, +y, +z
    blocks = []
    for d in range(3):
        if d == 0:
            m = ci < nx - 1
        elif d == 1:
            m = cj < ny - 1
        else:
            m = ck < nz - 1
        blocks.append((d, cid[m]))
    own_all, nb_all, verts_all = [], [], []
    for d, cells in blocks:
        i, j, k = cells % nx, (cells // nx) % ny, cells // (nx * ny)
        if d == 0:
            nb = cells + 1
            v = np.stack([p(i + 1, j, k), p(i + 1, j + 1, k), p(i + 1, j + 1, k + 1),
                          p(i + 1, j, k + 1)], axis=1)
        elif d == 1:
            nb = cells + nx
            v = np.stack([p(i, j + 1, k), p(i, j + 1, k + 1), p(i + 1, j + 1, k + 1),
                          p(i + 1, j + 1, k)], axis=1)
        else:
            nb = cells + nx * ny
            v = np.stack([p(i, j, k + 1), p(i + 1, j, k + 1), p(i + 1, j + 1, k + 1),
                          p(i, j + 1, k + 1)], axis=1)
        own_all.append(cells)
        nb_all.append(nb)
        verts_all.append(v)
    own = np.concatenate(own_all)
    nb = np.concatenate(nb_all)
    verts = np.concatenate(verts_all)
    order = np.lexsort((nb, own))
    own, nb, verts = own[order], nb[order], verts[order]

    if patch_types is None:
        patch_types = ["wall"] * 6
    names = ["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"]
    bown, bverts, patches = [], [], []
    start = own.shape[0]
    for side in range(6):
        d, hi = side // 2, side % 2
        if d == 0:
            cells = cid[ci == (nx - 1 if hi else 0)]
            i, j, k = cells % nx, (cells // nx) % ny, cells // (nx * ny)
            ii = i + hi
            v = np.stack([p(ii, j, k), p(ii, j + 1, k), p(ii, j + 1, k + 1), p(ii, j, k + 1)], 1)
        elif d == 1:
            cells = cid[cj == (ny - 1 if hi else 0)]
            i, j, k = cells % nx, (cells // nx) % ny, cells // (nx * ny)
            jj = j + hi
            v = np.stack([p(i, jj, k), p(i, jj, k + 1), p(i + 1, jj, k + 1), p(i + 1, jj, k)], 1)
        else:
            cells = cid[ck == (nz - 1 if hi else 0)]
            i, j, k = cells % nx, (cells // nx) % ny, cells // (nx * ny)
            kk = k + hi
            v = np.stack([p(i, j, kk), p(i + 1, j, kk), p(i + 1, j + 1, kk), p(i, j + 1, kk)], 1)
        if not hi:
            v = v[:, ::-1]  # outward normal on the low side
        bown.append(cells)
        bverts.append(v)
        patches.append((names[side], patch_types[side], start, int(cells.shape[0])))
        start += int(cells.shape[0])
    faces = np.concatenate([verts] + bverts).astype(np.int32)
    owner = np.concatenate([own] + bown).astype(np.int32)
    return PolyMesh(points=pts, faces=faces, nverts=np.full(faces.shape[0], 4, np.int32),
                    owner=owner, neighbour=nb.astype(np.int32), n_cells=C, patches=patches)


def uniform_box(nx, ny, nz, dx=1.0, origin=(0.0, 0.0, 0.0), patch_types=None) -> PolyMesh:
    ox, oy, oz = origin
    return hex_box(ox + dx * np.arange(nx + 1), oy + dx * np.arange(ny + 1),
                   oz + dx * np.arange(nz + 1), patch_types)


# Six tetrahedra per hex, all sharing the main diagonal v0-v6 of the cube
# (local vertex numbering v = i + 2 j + 4 k). Every hex face is then split
# along the diagonal through its lowest-index corner pair that the neighbour
# hex uses too, so faces conform across the mesh.
_TET6 = np.array([[0, 1, 3, 7], [0, 1, 7, 5], [0, 5, 7, 4],
                  [0, 3, 2, 7], [0, 2, 6, 7], [0, 6, 4, 7]], dtype=np.int64)


def jittered_tet_box(n, jitter=0.2, seed=0, dx=1.0, patch_types=None) -> PolyMesh:
    """n^3 hexes with interior nodes jittered uniformly by +-jitter*dx per axis
    (seeded PCG64), each hex split into 6 tetrahedra about a common diagonal.

    Faces are triangles; internal faces sorted by (owner, neighbour) with the
    normal pointing from owner to neighbour, boundary faces grouped per box side.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    g = dx * np.arange(n + 1, dtype=np.float64)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    P = np.stack([X, Y, Z], axis=-1)  # [i, j, k, 3]
    inner = (slice(1, n), slice(1, n), slice(1, n))
    P[inner] += rng.uniform(-jitter * dx, jitter * dx, size=P[inner].shape)
    pts = P.transpose(2, 1, 0, 3).reshape(-1, 3).astype(np.float32)
    pn = n + 1

    hid = np.arange(n ** 3, dtype=np.int64)
    hi, hj, hk = hid % n, (hid // n) % n, hid // (n * n)
    corners = np.stack([(hi + (v & 1)) + (hj + ((v >> 1) & 1)) * pn + (hk + (v >> 2)) * pn * pn
                        for v in range(8)], axis=1)  # [H, 8]
    tets = corners[:, _TET6].reshape(-1, 4)  # [6H, 4], cell id = 6 h + t
    T = tets.shape[0]
    P64 = pts.astype(np.float64)
    # orient every tet positively
    a, b, c, d = (P64[tets[:, q]] for q in range(4))
    vol6 = np.einsum("ij,ij->i", np.cross(b - a, c - a), d - a)
    neg = vol6 < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()

    # the 4 faces of each tet, opposite vertex 3,2,1,0; oriented outward
    fl = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], dtype=np.int64)
    tri = tets[:, fl].reshape(-1, 3)  # [4T, 3]
    cell = np.repeat(np.arange(T, dtype=np.int64), 4)
    key = np.sort(tri, axis=1)
    kk = key[:, 0] * pn ** 6 + key[:, 1] * pn ** 3 + key[:, 2]
    order = np.argsort(kk, kind="stable")
    ks = kk[order]
    same = np.zeros(ks.shape[0], dtype=bool)
    same[1:] = ks[1:] == ks[:-1]
    second = np.nonzero(same)[0]
    first = second - 1
    fa, fb = order[first], order[second]
    ca, cb = cell[fa], cell[fb]
    own = np.minimum(ca, cb)
    nbr = np.maximum(ca, cb)
    # keep the orientation of the owner's copy (outward from owner)
    own_tri = np.where((ca < cb)[:, None], tri[fa], tri[fb])
    o = np.lexsort((nbr, own))
    own, nbr, own_tri = own[o], nbr[o], own_tri[o]

    paired = np.zeros(tri.shape[0], dtype=bool)
    paired[fa] = True
    paired[fb] = True
    bidx = np.nonzero(~paired)[0]
    btri, bcell = tri[bidx], cell[bidx]
    cen = P64[btri].mean(axis=1)
    lo, hi_ = g[0], g[-1]
    tol = 1e-6 * dx
    side = np.full(bidx.shape[0], -1, dtype=np.int64)
    for s, (ax, val) in enumerate([(0, lo), (0, hi_), (1, lo), (1, hi_), (2, lo), (2, hi_)]):
        side[(side < 0) & (np.abs(cen[:, ax] - val) < tol)] = s
    assert (side >= 0).all()
    if patch_types is None:
        patch_types = ["wall"] * 6
    names = ["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"]
    bo = np.lexsort((bcell, side))
    btri, bcell, side = btri[bo], bcell[bo], side[bo]
    patches = []
    start = own.shape[0]
    for s in range(6):
        cnt = int((side == s).sum())
        patches.append((names[s], patch_types[s], start, cnt))
        start += cnt
    faces = np.concatenate([own_tri, btri]).astype(np.int32)
    owner = np.concatenate([own, bcell]).astype(np.int32)
    return PolyMesh(points=pts, faces=faces, nverts=np.full(faces.shape[0], 3, np.int32),
                    owner=owner, neighbour=nbr.astype(np.int32), n_cells=T, patches=patches)


# ----------------------------------------------------------------------------
# pre-processed mesh arrays (the solver's input)
# ----------------------------------------------------------------------------


@dataclass
class MeshArrays:
    n_cells: int
    n_faces: int
    n_internal: int
    owner: np.ndarray  # [F] int32
    neighbour: np.ndarray  # [F] int32 (boundary: n_cells + face - n_internal)
    face_area: np.ndarray  # [F]
    face_normal: np.ndarray  # [F, 3]
    face_centroid: np.ndarray  # [F, 3]
    streaming_dt: np.ndarray  # [F]
    cell_volume: np.ndarray  # [C + B]
    cell_centroid: np.ndarray  # [C + B, 3]
    stencil_offsets: np.ndarray  # [C + 1] int32
    stencil_cells: np.ndarray  # [nnz] int32
    stencil_faces: np.ndarray  # [nnz] int32
    bc_types: list

    @property
    def n_bc(self) -> int:
        return self.n_faces - self.n_internal

    @property
    def total_cells(self) -> int:
        return self.n_cells + self.n_bc


def _cross(b, c):
    return np.stack([b[:, 1] * c[:, 2] - b[:, 2] * c[:, 1],
                     b[:, 2] * c[:, 0] - b[:, 0] * c[:, 2],
                     b[:, 0] * c[:, 1] - b[:, 1] * c[:, 0]], axis=1)


def mesh_arrays(pm: PolyMesh, visc: float, gamma: float, fneq_min: float) -> MeshArrays:
    """The arrays unstructured_mesh.cpp computes from ``pm`` (see module doc)."""
    C, F, Fi = pm.n_cells, pm.n_faces, pm.n_internal
    B = F - Fi
    T = C + B
    P = pm.points.astype(np.float64)
    owner = pm.owner.astype(np.int64)
    nb = np.empty(F, dtype=np.int64)
    nb[:Fi] = pm.neighbour
    nb[Fi:] = C + np.arange(B)

    face_area = np.zeros(F)
    fc = np.zeros((F, 3))
    fn = np.zeros((F, 3))
    nvmax = int(pm.nverts.max())
    vol_idx, vol_val = [], []  # interleaved per face/triangle: owner +v, neighbour -v
    internal = np.arange(F) < Fi
    for t in range(nvmax - 2):
        has = pm.nverts > t + 2
        f = np.nonzero(has)[0]
        a = P[pm.faces[f, 0]]
        b = P[pm.faces[f, t + 1]]
        c = P[pm.faces[f, t + 2]]
        # tet_volume
        cr = _cross(b - a, c - a)
        vol = (a[:, 0] * cr[:, 0] + a[:, 1] * cr[:, 1] + a[:, 2] * cr[:, 2]) / 6
        vol_idx.append((f, t))
        vol_val.append(vol)
        # cell_tet_area
        d = np.stack([(a[:, 0] + b[:, 0] + c[:, 0]) / 3, (a[:, 1] + b[:, 1] + c[:, 1]) / 3,
                      (a[:, 2] + b[:, 2] + c[:, 2]) / 3], axis=1)
        cr2 = _cross(b - a, c - a)
        area = 0.5 * np.sqrt(cr2[:, 0] * cr2[:, 0] + cr2[:, 1] * cr2[:, 1] + cr2[:, 2] * cr2[:, 2])
        face_area[f] = face_area[f] + area
        d = d / (1 / area)[:, None]
        fc[f] = fc[f] + d
        fn[f] = fn[f] + cr2

    # cell volumes: face by face, triangle by triangle, the owner gains the
    # volume and the neighbour (internal faces only) loses it
    sf = np.concatenate([f for f, _t in vol_idx])
    st = np.concatenate([np.full(f.shape[0], t) for f, t in vol_idx])
    sv = np.concatenate(vol_val)
    o = np.lexsort((st, sf))
    sf, sv = sf[o], sv[o]
    is_int = internal[sf]
    idx = np.empty(sf.shape[0] * 2, dtype=np.int64)
    val = np.empty(sf.shape[0] * 2)
    keep = np.ones(sf.shape[0] * 2, dtype=bool)
    idx[0::2] = owner[sf]
    val[0::2] = sv
    idx[1::2] = np.where(is_int, nb[sf], 0)
    val[1::2] = -sv
    keep[1::2] = is_int
    cell_volume = np.zeros(T)
    np.add.at(cell_volume, idx[keep], val[keep])

    fmag = np.sqrt(fn[:, 0] ** 2 + fn[:, 1] ** 2 + fn[:, 2] ** 2)
    face_centroid = fc / face_area[:, None]
    face_normal = fn / fmag[:, None]
    with np.errstate(divide="ignore", invalid="ignore"):
        ref_dt = visc * 3 / gamma / fneq_min if fneq_min != 0 else math.inf
    sdt = 0.5 * np.sqrt(face_area)
    streaming_dt = np.where(ref_dt < sdt, ref_dt, sdt)

    # cell centroids: area-weighted face centroids, owner then neighbour per face
    idx = np.empty(F * 2, dtype=np.int64)
    keep = np.ones(F * 2, dtype=bool)
    idx[0::2] = owner
    idx[1::2] = np.where(internal, nb, 0)
    keep[1::2] = internal
    tca = np.zeros(T)
    cen = np.zeros((T, 3))
    area2 = np.repeat(face_area, 2)
    fc2 = np.repeat(fc, 2, axis=0)
    np.add.at(tca, idx[keep], area2[keep])
    for ax in range(3):
        np.add.at(cen[:, ax], idx[keep], fc2[keep, ax])
    cen[:C] = cen[:C] / tca[:C, None]
    # ghost centroids
    bf = np.arange(Fi, F)
    o_c = cen[owner[bf]]
    rel = (face_centroid[bf] - o_c) / 0.5
    cen[C:] = o_c + rel * np.abs(face_normal[bf])

    # gradient stencil: walking the faces in order, an internal face appends
    # the neighbour to the owner's list and the owner to the neighbour's; a
    # boundary face appends the ghost to the owner's list
    src = np.concatenate([np.stack([owner[:Fi], nb[:Fi]], 1).ravel(), owner[Fi:]])
    dst = np.concatenate([np.stack([nb[:Fi], owner[:Fi]], 1).ravel(), nb[Fi:]])
    fid = np.concatenate([np.repeat(np.arange(Fi), 2), np.arange(Fi, F)])
    o = np.argsort(src, kind="stable")
    ent_cell, ent_face = dst[o], fid[o]
    off = np.zeros(C + 1, dtype=np.int64)
    off[1:] = np.cumsum(np.bincount(src, minlength=C))

    return MeshArrays(n_cells=C, n_faces=F, n_internal=Fi, owner=owner.astype(np.int32),
                      neighbour=nb.astype(np.int32), face_area=face_area,
                      face_normal=face_normal, face_centroid=face_centroid,
                      streaming_dt=streaming_dt, cell_volume=cell_volume, cell_centroid=cen,
                      stencil_offsets=off.astype(np.int32),
                      stencil_cells=ent_cell.astype(np.int32),
                      stencil_faces=ent_face.astype(np.int32), bc_types=pm.bc_types())


# ----------------------------------------------------------------------------
# Lagrangian nodes
# ----------------------------------------------------------------------------


def fibonacci_sphere(n, radius, centre):
    """n points on a sphere by the golden-angle (Fibonacci) lattice, in order of
    decreasing z. Spacing ~ sqrt(4 pi r^2 / n)."""
    i = np.arange(n, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = i * (math.pi * (3.0 - math.sqrt(5.0)))
    pts = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1) * radius
    return pts + np.asarray(centre, dtype=np.float64)[None, :]


def write_spring_network(path, pts):
    """Node file in the layout lagrangian_object::mesh_read reads
    (lagrangian_object.cpp:116-213): counts, xyz per node, no tets, no springs,
    zero neighbours per node."""
    with open(path, "w") as f:
        f.write("%d 0 0\n" % pts.shape[0])
        for x, y, z in pts:
            f.write("%.17g %.17g %.17g\n" % (x, y, z))
        for _ in range(pts.shape[0]):
            f.write("0\n")


# ----------------------------------------------------------------------------
# polyMesh + XML writers (for running the reference program on a case)
# ----------------------------------------------------------------------------

_BANNER = """/*--------------------------------*- C++ -*----------------------------------*\\
  =========                 |
  \\\\      /  F ield         | OpenFOAM: The Open Source CFD Toolbox
   \\\\    /   O peration     | Version:  synthetic
    \\\\  /    A nd           | Web:      www.OpenFOAM.org
     \\\\/     M anipulation  |
\\*---------------------------------------------------------------------------*/
"""


def _header(cls, obj, note=None):
    s = _BANNER + "FoamFile\n{\n    version     2.0;\n    format      ascii;\n"
    s += "    class       %s;\n" % cls
    s += '    note        "%s";\n' % (note or "")
    s += '    location    "constant/polyMesh";\n    object      %s;\n}\n' % obj
    return s


def write_polymesh(dirpath, pm: PolyMesh):
    """Write points/faces/owner/neighbour/boundary. The owner header carries the
    nPoints/nCells/nFaces/nInternalFaces note on line 12, where
    unstructured_mesh::import_openfoam_mesh reads it (unstructured_mesh.cpp:273)."""
    os.makedirs(dirpath, exist_ok=True)
    P, F, C, Fi = pm.points.shape[0], pm.n_faces, pm.n_cells, pm.n_internal
    note = "nPoints:%d nCells:%d nFaces:%d nInternalFaces:%d" % (P, C, F, Fi)
    with open(os.path.join(dirpath, "owner"), "w") as f:
        f.write(_header("labelList", "owner", note))
        f.write("\n%d\n(\n" % F)
        f.write("\n".join(map(str, np.asarray(pm.owner).tolist())))
        f.write("\n)\n")
    with open(os.path.join(dirpath, "neighbour"), "w") as f:
        f.write(_header("labelList", "neighbour", note))
        f.write("\n%d\n(\n" % Fi)
        f.write("\n".join(map(str, np.asarray(pm.neighbour).tolist())))
        f.write("\n)\n")
    with open(os.path.join(dirpath, "points"), "w") as f:
        f.write(_header("vectorField", "points"))
        f.write("\n%d\n(\n" % P)
        # %.9g of each coordinate as a Python float (the points are float32)
        f.write("\n".join(map("(%.9g %.9g %.9g)".__mod__,
                              map(tuple, np.asarray(pm.points, np.float64).tolist()))))
        f.write("\n)\n")
    with open(os.path.join(dirpath, "faces"), "w") as f:
        f.write(_header("faceList", "faces"))
        f.write("\n%d\n(\n" % F)
        nverts = np.asarray(pm.nverts).tolist()
        rows = np.asarray(pm.faces).tolist()
        fmt = {}
        for n in set(nverts):
            fmt[n] = ("%d(" % n + " ".join(["%d"] * n) + ")").__mod__
        f.write("\n".join(fmt[n](tuple(row[:n])) for row, n in zip(rows, nverts)))
        f.write("\n)\n")
    with open(os.path.join(dirpath, "boundary"), "w") as f:
        f.write(_header("polyBoundaryMesh", "boundary"))
        f.write("\n%d\n(\n" % len(pm.patches))
        for name, ptype, start, n in pm.patches:
            f.write("    %s\n    {\n        type %s;\n        nFaces %d;\n        startFace %d;\n    }\n"
                    % (name, ptype, n, start))
        f.write(")\n")


@dataclass
class BC:
    name: str  # the patch type string it applies to
    rho: float
    u: float
    v: float
    w: float
    vel_type: str  # a name of BC_TYPES
    rho_type: str  # a name of BC_TYPES


@dataclass
class Case:
    """Everything the reference's XML holds for an unstructured run."""

    mesh_dir: str
    X: float
    Y: float
    Z: float
    streaming_dt: float = 0.5
    ref_length: float = 1.0
    origin: tuple = (0.0, 0.0, 0.0)
    reynolds: float = 100.0
    mach: float = 0.1  # max velocity (lattice units)
    scale: float = 1.0
    tolerance: float = 1e-12
    gamma: float = 1.0
    steps: int = 10
    dt: float = 0.1  # time_marching_step
    gradient_calc: str = "LS"
    fneq_min: float = 0.0
    output_dir: str = "out/"
    output_step: int = 1000000
    restart: bool = False
    gpu_solver: int = 1
    average_rho: float = 1.0
    pressure_gradient: float = 0.0
    rho0: float = 1.0
    u0: float = 0.0
    bcs: list = field(default_factory=list)
    obj_nodes_file: str = ""
    obj_num_nodes: int = 1
    obj_radius: float = 1.0
    obj_depth: float = 1.0
    obj_stiffness: float = 0.0
    obj_centre: tuple = (0.0, 0.0, 0.0)

    @property
    def visc(self) -> float:
        """global_variables::initialise: nu = U L / Re (global_variables.cpp:24)."""
        return self.mach * self.ref_length / self.reynolds

    def bc_factor(self) -> float:
        """XML velocities are scaled by mach/scale (preprocessor.cpp:187-190)."""
        return self.mach / self.scale


def write_xml(path, c: Case):
    """The case XML in the layout preprocessor.cpp parses. The root element must
    be the document's first child (no <?xml?> declaration, preprocessor.cpp:520)
    and the legacy <boundary_conditions> block must exist (:304-434)."""
    g = []
    add = g.append
    add("<plfbs_case>")
    add(" <global_variables>")
    for k, v in [("tolerance", "%.17g" % c.tolerance), ("pre_condition_gamma", "%.17g" % c.gamma),
                 ("simulation_length", "%d" % c.steps), ("time_marching_step", "%.17g" % c.dt),
                 ("reynolds_no", "%.17g" % c.reynolds), ("mach_no", "%.17g" % c.mach),
                 ("simulation_name", "case"), ("output_directory", c.output_dir),
                 ("max_multi_grid_levels", "0"), ("FMG_levels", "0"), ("FMG_tolerance", "0"),
                 ("dissipation_kappa_2", "0"), ("dissipation_kappa_4", "0"),
                 ("martinelli_exponent", "0"), ("testcase", "0"), ("mesh_type", "3"),
                 ("scale", "%.17g" % c.scale), ("womersley_no", "0"),
                 ("output_step", "%d" % c.output_step), ("import_file", c.mesh_dir.rstrip("/") + "/"),
                 ("import_format", "openfoam"), ("gradient_calc", c.gradient_calc),
                 ("restart_analysis", "true" if c.restart else "false"),
                 ("time_stepping", "constant"), ("preconditioning", "false"),
                 ("gpu_solver", "%d" % c.gpu_solver), ("fneq_min", "%.17g" % c.fneq_min)]:
        add("  <%s>%s</%s>" % (k, v, k))
    add(" </global_variables>")
    add(" <geometry>")
    for k, v in [("x", c.X), ("y", c.Y), ("z", c.Z), ("dx", 1.0), ("dy", 1.0), ("dz", 1.0),
                 ("streaming_dt", c.streaming_dt), ("origin_x", c.origin[0]),
                 ("origin_y", c.origin[1]), ("origin_z", c.origin[2]),
                 ("ref_length", c.ref_length)]:
        add("  <%s>%.17g</%s>" % (k, v, k))
    add(" </geometry>")
    add(" <initial_conditions>")
    add("  <average_rho>%.17g</average_rho>" % c.average_rho)
    add("  <pressure_gradient>%.17g</pressure_gradient>" % c.pressure_gradient)
    add("  <rho><gradient><x>0</x><y>0</y><z>0</z></gradient>"
        "<origin_magnitude><x>%.17g</x><y>0</y><z>0</z></origin_magnitude></rho>" % c.rho0)
    add("  <origin_location><x>0</x><y>0</y><z>0</z></origin_location>")
    add("  <vel><gradient><x>0</x><y>0</y><z>0</z></gradient>"
        "<origin_magnitude><x>%.17g</x><y>0</y><z>0</z></origin_magnitude></vel>" % c.u0)
    add("  <u>0</u><v>0</v><w>0</w>")
    add(" </initial_conditions>")
    add(" <boundary_conditions>")
    for side in ("west", "east", "north", "south"):
        add("  <%s><rho>1</rho><u>0</u><v>0</v><vel_type>dirichlet</vel_type>"
            "<rho_type>neumann</rho_type></%s>" % (side, side))
    add(" </boundary_conditions>")
    add(" <uns_boundary_conditions>")
    for b in c.bcs:
        add("  <bc><name>%s</name><rho>%.17g</rho><u>%.17g</u><v>%.17g</v><w>%.17g</w>"
            "<vel_type>%s</vel_type><rho_type>%s</rho_type></bc>"
            % (b.name, b.rho, b.u, b.v, b.w, b.vel_type, b.rho_type))
    add("  <periodic_translation><x>0</x><y>0</y><z>0</z></periodic_translation>")
    add(" </uns_boundary_conditions>")
    add(" <lagrangian_objects>")
    add("  <object><name>body</name><num_nodes>%d</num_nodes><radius>%.17g</radius>"
        "<depth>%.17g</depth><stiffness>%.17g</stiffness><centre_x>%.17g</centre_x>"
        "<centre_y>%.17g</centre_y><centre_z>%.17g</centre_z><type>spring_network</type>"
        "<mesh_file>%s</mesh_file></object>"
        % (c.obj_num_nodes, c.obj_radius, c.obj_depth, c.obj_stiffness, c.obj_centre[0],
           c.obj_centre[1], c.obj_centre[2], c.obj_nodes_file))
    add(" </lagrangian_objects>")
    add("</plfbs_case>")
    with open(path, "w") as f:
        f.write("\n".join(g) + "\n")


# The reference's boundary-type names and codes, the same table for velocity
# and density (preprocessor.cpp:241-262). The GPU path defines 1, 2 and 9
# (LBFS.cu:1252-1294); the CPU Solver 1, 2, 3, 6, 7 and 8 (Solution.cpp:759-833,
# gradients.cpp:395-506).
BC_TYPES = {"dirichlet": 1, "neumann": 2, "periodic": 3, "parabolic-N": 4, "parabolic-W": 5,
            "inlet": 6, "wall": 7, "symmetry-x": 8, "parabolic": 9}
VEL_TYPES = BC_TYPES
RHO_TYPES = BC_TYPES


def bc_arrays(ma: MeshArrays, case: Case):
    """Per boundary face (rho_type, vel_type, [u, v, w, rho]) as
    Boundary_Conditions::assign_boundary_conditions builds them
    (Boundary_Conditions.cpp:388-452): the patch type string selects the XML
    <bc> with that name; velocities carry the mach/scale factor."""
    by_name = {b.name: b for b in case.bcs}
    fac = case.bc_factor()
    B = ma.n_bc
    rt = np.zeros(B, np.int32)
    vt = np.zeros(B, np.int32)
    val = np.zeros((B, 4))
    for i, t in enumerate(ma.bc_types):
        b = by_name[t]
        rt[i] = RHO_TYPES[b.rho_type]
        vt[i] = VEL_TYPES[b.vel_type]
        val[i] = (b.u * fac, b.v * fac, b.w * fac, b.rho)
    return rt, vt, val
