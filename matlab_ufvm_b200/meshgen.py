"""Seeded synthetic case generators that emit OpenFOAM-ordered polyMesh data.

Face ordering follows OpenFOAM's polyMesh convention, which is what uFVM's reader
(``src/utilities/IO/cfdReadPolyMesh.m:25-214``) consumes:

* interior faces first, upper-triangular: ``owner < neighbour``, sorted by owner then
  neighbour, normal pointing from owner to neighbour;
* boundary faces afterwards, grouped by patch, normal pointing out of the domain.

Indices are 0-based here; the reference converts to 1-based on read.

Generators:

* :func:`cavity_hex` -- n_x x n_y x n_z hex box (2D cases use one cell in z with an
  ``empty`` front/back patch), laid out exactly like blockMesh lays out uFVM's
  ``tutorials/incompressible/movingLid`` mesh (same points, node order and patch order).
* :func:`channel_tet` -- box split into hexes, each hex cut into 6 tets (Freudenthal /
  Kuhn split along the main diagonal), interior nodes jittered by U(-a h, a h) from a
  seeded generator, boundary nodes fixed.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np


@dataclass
class Patch:
    name: str
    type: str          # 'wall' | 'inlet' | 'outlet' | 'symmetry' | 'empty'
    start: int         # first face (0-based)
    n: int             # number of faces


@dataclass
class PolyMesh:
    points: np.ndarray                 # (nP, 3) float64
    face_start: np.ndarray             # (F+1,) int32, CSR offsets into face_nodes
    face_nodes: np.ndarray             # (sum,) int32, 0-based point ids
    owner: np.ndarray                  # (F,) int32
    neighbour: np.ndarray              # (Fi,) int32
    patches: List[Patch] = field(default_factory=list)

    @property
    def n_faces(self) -> int:
        return int(self.owner.shape[0])

    @property
    def n_interior(self) -> int:
        return int(self.neighbour.shape[0])

    @property
    def n_cells(self) -> int:
        m = int(self.owner.max()) + 1
        if self.neighbour.size:
            m = max(m, int(self.neighbour.max()) + 1)
        return m

    def patch(self, name: str) -> Patch:
        for p in self.patches:
            if p.name == name:
                return p
        raise KeyError(name)


def _text_round(x: np.ndarray, digits: int) -> np.ndarray:
    """Round coordinates the way an ASCII polyMesh round-trip does (``%.{digits}g``)."""
    if digits <= 0:
        return x
    f = np.vectorize(lambda v: float(f"{v:.{digits}g}"), otypes=[np.float64])
    return f(x)


def cavity_hex(nx: int, ny: int, nz: int = 1, lx: float = 1.0, ly: float = 1.0,
               lz: float = 0.1, digits: int = 12, two_d: bool | None = None) -> PolyMesh:
    """Lid-driven cavity box.

    Patches: ``movingWall`` (y = ly), ``fixedWalls`` (x = 0, x = lx, y = 0 and, in 3D,
    z = 0, z = lz) and, in 2D (``nz == 1``), ``frontAndBack`` (empty).
    With ``nx = ny = 20, nz = 1, lx = ly = 0.1, lz = 0.01, digits = 6`` the result is
    byte-for-byte the polyMesh of uFVM's ``movingLid`` / ``cavity1`` tutorials.
    """
    if two_d is None:
        two_d = nz == 1
    px, py, pz = nx + 1, ny + 1, nz + 1
    i = np.arange(px, dtype=np.float64)
    j = np.arange(py, dtype=np.float64)
    k = np.arange(pz, dtype=np.float64)
    zz, yy, xx = np.meshgrid(k, j, i, indexing="ij")
    pts = np.stack([xx.ravel() * (lx / nx), yy.ravel() * (ly / ny), zz.ravel() * (lz / nz)], axis=1)
    pts = _text_round(pts, digits)

    def P(ii, jj, kk):
        return ii + px * jj + px * py * kk

    def C(ii, jj, kk):
        return ii + nx * jj + nx * ny * kk

    faces: List[Tuple[int, int, int, int]] = []
    owner: List[int] = []
    neigh: List[int] = []
    # interior faces, per owner cell: +x, +y, +z (ascending neighbour index)
    for kk in range(nz):
        for jj in range(ny):
            for ii in range(nx):
                c = C(ii, jj, kk)
                if ii + 1 < nx:
                    faces.append((P(ii + 1, jj, kk), P(ii + 1, jj + 1, kk), P(ii + 1, jj + 1, kk + 1), P(ii + 1, jj, kk + 1)))
                    owner.append(c); neigh.append(C(ii + 1, jj, kk))
                if jj + 1 < ny:
                    faces.append((P(ii, jj + 1, kk), P(ii, jj + 1, kk + 1), P(ii + 1, jj + 1, kk + 1), P(ii + 1, jj + 1, kk)))
                    owner.append(c); neigh.append(C(ii, jj + 1, kk))
                if kk + 1 < nz:
                    faces.append((P(ii, jj, kk + 1), P(ii + 1, jj, kk + 1), P(ii + 1, jj + 1, kk + 1), P(ii, jj + 1, kk + 1)))
                    owner.append(c); neigh.append(C(ii, jj, kk + 1))
    patches: List[Patch] = []

    def add_patch(name, ptype, items):
        start = len(faces)
        for f, o in items:
            faces.append(f); owner.append(o)
        patches.append(Patch(name, ptype, start, len(faces) - start))

    # movingWall: y = ly
    top = []
    for kk in range(nz):
        for ii in range(nx):
            top.append(((P(ii, ny, kk), P(ii, ny, kk + 1), P(ii + 1, ny, kk + 1), P(ii + 1, ny, kk)), C(ii, ny - 1, kk)))
    add_patch("movingWall", "wall", top)
    walls = []
    for kk in range(nz):  # left x = 0
        for jj in range(ny):
            walls.append(((P(0, jj, kk), P(0, jj, kk + 1), P(0, jj + 1, kk + 1), P(0, jj + 1, kk)), C(0, jj, kk)))
    for kk in range(nz):  # right x = lx
        for jj in range(ny):
            walls.append(((P(nx, jj, kk), P(nx, jj + 1, kk), P(nx, jj + 1, kk + 1), P(nx, jj, kk + 1)), C(nx - 1, jj, kk)))
    for kk in range(nz):  # bottom y = 0
        for ii in range(nx):
            walls.append(((P(ii, 0, kk), P(ii + 1, 0, kk), P(ii + 1, 0, kk + 1), P(ii, 0, kk + 1)), C(ii, 0, kk)))
    zfaces_lo = []
    zfaces_hi = []
    for ii in range(nx):  # blockMesh order for the z faces: i-major, j-minor
        for jj in range(ny):
            zfaces_lo.append(((P(ii, jj, 0), P(ii, jj + 1, 0), P(ii + 1, jj + 1, 0), P(ii + 1, jj, 0)), C(ii, jj, 0)))
    for ii in range(nx):
        for jj in range(ny):
            zfaces_hi.append(((P(ii, jj, nz), P(ii + 1, jj, nz), P(ii + 1, jj + 1, nz), P(ii, jj + 1, nz)), C(ii, jj, nz - 1)))
    if two_d:
        add_patch("fixedWalls", "wall", walls)
        add_patch("frontAndBack", "empty", zfaces_lo + zfaces_hi)
    else:
        add_patch("fixedWalls", "wall", walls + zfaces_lo + zfaces_hi)
    fn = np.asarray(faces, dtype=np.int32)
    return PolyMesh(points=pts,
                    face_start=np.arange(0, 4 * len(faces) + 1, 4, dtype=np.int32),
                    face_nodes=fn.ravel(),
                    owner=np.asarray(owner, dtype=np.int32),
                    neighbour=np.asarray(neigh, dtype=np.int32),
                    patches=patches)


# Freudenthal split: for each permutation (a, b, c) of the axes the tet
# (v0, v0 + e_a, v0 + e_a + e_b, v0 + e_a + e_b + e_c).
_PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def channel_tet(nx: int = 140, ny: int = 35, nz: int = 35, lx: float = 4.0, ly: float = 1.0,
                lz: float = 1.0, jitter: float = 0.2, seed: int = 12345) -> PolyMesh:
    """Jittered 6-tet channel. Patches: ``inlet`` (x = 0), ``outlet`` (x = lx), ``walls``."""
    px, py, pz = nx + 1, ny + 1, nz + 1
    hx, hy, hz = lx / nx, ly / ny, lz / nz
    kk, jj, ii = np.meshgrid(np.arange(pz), np.arange(py), np.arange(px), indexing="ij")
    ii = ii.ravel(); jj = jj.ravel(); kk = kk.ravel()
    pts = np.stack([ii * hx, jj * hy, kk * hz], axis=1).astype(np.float64)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-jitter, jitter, size=pts.shape) * np.array([hx, hy, hz])
        interior = (ii > 0) & (ii < nx) & (jj > 0) & (jj < ny) & (kk > 0) & (kk < nz)
        pts[interior] += d[interior]

    def P(a, b, c):
        return a + px * b + px * py * c

    hk, hj, hi = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    hi = hi.ravel(); hj = hj.ravel(); hk = hk.ravel()
    nh = hi.size
    tets = np.empty((nh, 6, 4), dtype=np.int64)
    for t, perm in enumerate(_PERMS):
        off = np.zeros((nh, 3), dtype=np.int64)
        verts = [P(hi, hj, hk)]
        for ax in perm:
            off[:, ax] += 1
            verts.append(P(hi + off[:, 0], hj + off[:, 1], hk + off[:, 2]))
        tets[:, t, :] = np.stack(verts, axis=1)
    tets = tets.reshape(-1, 4)
    # odd permutations give negatively oriented tets; swap two nodes so all are positive
    neg = np.repeat(np.array([((p[0] - p[1]) * (p[1] - p[2]) * (p[2] - p[0])) < 0 for p in _PERMS]), 1)
    tets = tets.reshape(nh, 6, 4)
    tets[:, neg, 1], tets[:, neg, 2] = tets[:, neg, 2].copy(), tets[:, neg, 1].copy()
    tets = tets.reshape(-1, 4)
    a, b, c, dd = (pts[tets[:, q]] for q in range(4))
    vol = np.einsum("ij,ij->i", np.cross(b - a, c - a), dd - a)
    if np.any(vol <= 0):
        raise ValueError(f"{int(np.sum(vol <= 0))} inverted tets; reduce jitter")
    # all 4 faces of every tet (opposite vertex q)
    fidx = np.array([[1, 2, 3], [0, 3, 2], [0, 1, 3], [0, 2, 1]])
    tri = tets[:, fidx].reshape(-1, 3)                 # (4nc, 3)
    nc = tets.shape[0]
    cell = np.repeat(np.arange(nc, dtype=np.int64), 4)
    key = np.sort(tri, axis=1)
    order = np.lexsort((key[:, 2], key[:, 1], key[:, 0]))
    key_s = key[order]
    same = np.all(key_s[1:] == key_s[:-1], axis=1)
    # pairs (interior): positions order[p], order[p+1] where same[p]
    pidx = np.nonzero(same)[0]
    fa = order[pidx]; fb = order[pidx + 1]
    ca = cell[fa]; cb = cell[fb]
    own = np.minimum(ca, cb); nei = np.maximum(ca, cb)
    own_face = np.where(ca < cb, fa, fb)
    paired = np.zeros(tri.shape[0], dtype=bool)
    paired[fa] = True; paired[fb] = True
    ib = np.nonzero(~paired)[0]
    cent = pts[tets].mean(axis=1)

    def orient(tri_nodes, own_cells):
        p0 = pts[tri_nodes[:, 0]]; p1 = pts[tri_nodes[:, 1]]; p2 = pts[tri_nodes[:, 2]]
        nrm = np.cross(p1 - p0, p2 - p0)
        fc = (p0 + p1 + p2) / 3.0
        s = np.einsum("ij,ij->i", nrm, fc - cent[own_cells])
        out = tri_nodes.copy()
        flip = s < 0
        out[flip] = out[flip][:, [0, 2, 1]]
        return out

    itri = orient(tri[own_face], own)
    o2 = np.lexsort((nei, own))
    itri = itri[o2]; own = own[o2]; nei = nei[o2]
    btri = orient(tri[ib], cell[ib])
    bown = cell[ib]
    # boundary nodes are not jittered, so a boundary face lies exactly on its plane
    x0 = np.all(pts[btri][:, :, 0] == 0.0, axis=1)
    x1 = np.all(pts[btri][:, :, 0] == pts[:, 0].max(), axis=1)
    is_in = x0; is_out = x1
    is_wall = ~(is_in | is_out)
    faces = [itri]; owners = [own]
    patches: List[Patch] = []
    start = itri.shape[0]
    for name, ptype, m in (("inlet", "inlet", is_in), ("outlet", "outlet", is_out), ("walls", "wall", is_wall)):
        sel = np.nonzero(m)[0]
        s2 = sel[np.lexsort((btri[sel].min(axis=1), bown[sel]))]
        faces.append(btri[s2]); owners.append(bown[s2])
        patches.append(Patch(name, ptype, start, int(s2.size)))
        start += int(s2.size)
    fn = np.concatenate(faces).astype(np.int32)
    return PolyMesh(points=pts,
                    face_start=np.arange(0, 3 * fn.shape[0] + 1, 3, dtype=np.int32),
                    face_nodes=fn.ravel(),
                    owner=np.concatenate(owners).astype(np.int32),
                    neighbour=nei.astype(np.int32),
                    patches=patches)
