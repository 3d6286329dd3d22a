"""CPU oracle for HyTeG's matrix-free P1 multigrid path.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``hyteg_b200`` product imports this
module; it is used by ``tests/``, ``__graft_entry__.smoke()`` and the CPU leg
of ``bench.py`` as the checker.

What it restates (reference paths are relative to the hyteg source tree):

* Primitive ordering and local orientation of a macro mesh:
  ``src/hyteg/mesh/MeshInfo.cpp`` (``addEdge``/``addFace`` sort the vertex ids,
  cells keep the mesh order) and
  ``src/hyteg/primitivestorage/SetupPrimitiveStorage.cpp:130-412`` (ids are
  generated vertex -> edge -> face -> cell in map order; face vertex order is
  the sorted order; cell local edges/faces at :305-315).
* Boundary flags: ``SetupPrimitiveStorage.cpp:977-988,1092-1150``
  (``setMeshBoundaryFlagsOnBoundary``/``onBoundary``).
* Vertex-DoF memory layout per primitive and level:
  ``src/hyteg/p1functionspace/VertexDoFMemory.hpp:39-60``,
  ``src/hyteg/indexing/MacroCellIndexing.hpp:39-52``,
  ``src/hyteg/indexing/MacroFaceIndexing.hpp:39-50``.
* Micro-cells of a refined macro-cell:
  ``src/hyteg/volumedofspace/CellDoFIndexing.hpp:64-198``;
  micro-vertex coordinates ``src/hyteg/p1functionspace/VertexDoFMacroCell.hpp:70-77``.
* P1 Laplace element matrix (FEniCS form ``p1_tet_diffusion``,
  ``src/hyteg/forms/form_fenics_generated/p1_tet_diffusion.h``):
  K = |det J| / 6 * G G^T.
* ``P1Operator::apply`` (``src/hyteg/p1functionspace/P1Operator.hpp:192-320``):
  y = A x on owned DoFs whose boundary type matches ``flag``.  The oracle
  assembles A from micro-cell element matrices over HyTeG's own layout
  instead of going through stencils and ghost layers: every P1 stencil entry
  of HyTeG is a sum of element-matrix entries over the micro-cells around a
  micro-vertex (``src/hyteg/p1functionspace/P1Elements.hpp:466-529``), so the
  two agree up to rounding of the summation order.
* ``P1toP1LinearRestriction::restrict3D`` (``P1toP1LinearRestriction.cpp:169-346``)
  through the generated pull kernel ``restrict_3D_macrocell_P1_pull_additive``:
  per macro-cell pull with weights 1 and 1/2, each fine value scaled by
  1/(number of macro-cells around the primitive owning that fine point), then
  additive communication into flagged owners.
* ``P1toP1LinearProlongation::prolongate3DAdditively``
  (``P1toP1LinearProlongation.cpp:194-410``): linear interpolation added to
  (or replacing) flagged owned fine DoFs.
* ``WeightedJacobiSmoother::solve`` (``solvers/WeightedJacobiSmoother.hpp:46-66``)
  with ``P1Operator::smooth_jac`` (``P1Operator.hpp:429-447``).
* ``ChebyshevSmoother::solve`` (``solvers/ChebyshevSmoother.hpp:112-240``),
  coefficients (``:329-555``), ``chebyshev::estimateRadius`` (``:656-676``)
  and ``estimateSpectralRadiusWithPowerIteration``
  (``numerictools/SpectrumEstimation.hpp:56-84``).
* ``CGSolver::solve`` (``solvers/CGSolver.hpp:94-206``).
* ``GeometricMultigridSolver::solveRecursively``
  (``solvers/GeometricMultigridSolver.hpp:207-305``).

Vectors are HyTeG layout buffers of one level (all primitives packed in the
order vertices, edges, faces, cells, each with its full HyTeG array including
ghost layers).  Only owned slots carry meaning; copy slots can be filled with
``Level.sync``.
"""

from __future__ import annotations

import itertools
import math
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

INNER = 1
DIRICHLET = 2
NEUMANN = 4
FREESLIP = 8
ALL = INNER | DIRICHLET | NEUMANN | FREESLIP

# 14 neighbour directions of the 3D P1 stencil
# (src/hyteg/p1functionspace/VertexDoFIndexing.hpp:289-323).
STENCIL_DIRS = np.array(
    [
        (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1),
        (-1, 1, 0), (1, -1, 0), (-1, 0, 1), (1, 0, -1), (0, -1, 1), (0, 1, -1),
        (1, -1, 1), (-1, 1, -1),
    ],
    dtype=np.int64,
)

# Micro-cell types: vertex offsets and row width (number of micro-edges per
# edge minus the shift), CellDoFIndexing.hpp:64-198.
MICRO_CELL_TYPES = [
    ("WHITE_UP", [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)], 0),
    ("BLUE_UP", [(1, 0, 0), (1, 1, 0), (0, 1, 0), (1, 0, 1)], 1),
    ("GREEN_UP", [(1, 0, 0), (0, 1, 0), (1, 0, 1), (0, 0, 1)], 1),
    ("WHITE_DOWN", [(1, 1, 0), (1, 1, 1), (0, 1, 1), (1, 0, 1)], 2),
    ("BLUE_DOWN", [(1, 0, 1), (0, 1, 1), (0, 0, 1), (0, 1, 0)], 1),
    ("GREEN_DOWN", [(0, 1, 0), (1, 1, 0), (1, 0, 1), (0, 1, 1)], 1),
]


def tet_size(w):
    """linearMacroCellSize (MacroCellIndexing.hpp:39-42)."""
    return ((w + 2) * (w + 1) * w) // 6


def tri_size(w):
    """linearMacroFaceSize (MacroFaceIndexing.hpp:39-42)."""
    return ((w + 1) * w) // 2


def cell_index(n, x, y, z):
    """linearMacroCellIndex with width n+1 (MacroCellIndexing.hpp:45-52)."""
    w = n + 1
    wz = w - z
    slice_off = tet_size(w) - ((wz + 2) * (wz + 1) * wz) // 6
    row_off = y * (wz + 1) - ((y + 1) * y) // 2
    return slice_off + row_off + x


def face_index(n, i, j):
    """linearMacroFaceIndex with width n+1 (MacroFaceIndexing.hpp:45-50)."""
    w = n + 1
    return j * (w + 1) - ((j + 1) * j) // 2 + i


def tet_points(w):
    """All (x, y, z) with x+y+z <= w-1, in HyTeG memory order (z-major, then y, then x)."""
    if w <= 0:
        return np.zeros((0, 3), dtype=np.int64)
    zr = np.repeat(np.arange(w, dtype=np.int64), w - np.arange(w))  # one entry per row (y, z)
    yr = np.concatenate([np.arange(w - z, dtype=np.int64) for z in range(w)])
    lens = w - zr - yr
    z = np.repeat(zr, lens)
    y = np.repeat(yr, lens)
    x = np.arange(z.size, dtype=np.int64) - np.repeat(np.cumsum(lens) - lens, lens)
    return np.stack([x, y, z], axis=1)


class MacroMesh:
    """Macro-primitive topology with HyTeG's id order and local orientations."""

    def __init__(self, coords, tets, boundary_flag=1, inner_flag=0, bc_types=None):
        coords = np.asarray(coords, dtype=np.float64)
        self.vcoords = coords
        nv = coords.shape[0]
        cells = sorted(tuple(int(v) for v in t) for t in tets)  # std::map keyed by vertex list
        edge_set, face_set = set(), set()
        for c in cells:
            for a, b in itertools.combinations(c, 2):
                edge_set.add(tuple(sorted((a, b))))
            for tri in itertools.combinations(c, 3):
                face_set.add(tuple(sorted(tri)))
        self.edges = sorted(edge_set)
        self.faces = sorted(face_set)
        self.cells = cells
        self.edge_id = {e: i for i, e in enumerate(self.edges)}
        self.face_id = {f: i for i, f in enumerate(self.faces)}
        nE, nF, nC = len(self.edges), len(self.faces), len(self.cells)
        self.nV, self.nE, self.nF, self.nC = nv, nE, nF, nC
        # neighbour lists in insertion order
        self.v_edges = [[] for _ in range(nv)]
        self.v_faces = [[] for _ in range(nv)]
        self.v_cells = [[] for _ in range(nv)]
        self.e_faces = [[] for _ in range(nE)]
        self.e_cells = [[] for _ in range(nE)]
        self.f_cells = [[] for _ in range(nF)]
        for i, (a, b) in enumerate(self.edges):
            self.v_edges[a].append(i)
            self.v_edges[b].append(i)
        for i, f in enumerate(self.faces):
            for v in f:
                self.v_faces[v].append(i)
            for e in itertools.combinations(f, 2):
                self.e_faces[self.edge_id[e]].append(i)
        # cell local edges / faces (SetupPrimitiveStorage.cpp:305-315)
        self.cell_edges, self.cell_faces = [], []
        for ci, c in enumerate(cells):
            v0, v1, v2, v3 = c
            ce = [self.edge_id[tuple(sorted(p))] for p in ((v0, v1), (v0, v2), (v1, v2), (v0, v3), (v1, v3), (v2, v3))]
            cf = [self.face_id[tuple(sorted(t))] for t in ((v0, v1, v2), (v0, v1, v3), (v0, v2, v3), (v1, v2, v3))]
            self.cell_edges.append(ce)
            self.cell_faces.append(cf)
            for v in c:
                self.v_cells[v].append(ci)
            for e in ce:
                self.e_cells[e].append(ci)
            for f in cf:
                self.f_cells[f].append(ci)
        # boundary flags (setMeshBoundaryFlagsOnBoundary(boundary_flag, inner_flag, true))
        f_bnd = [len(self.f_cells[f]) == 1 for f in range(nF)]
        e_bnd = [any(f_bnd[f] for f in self.e_faces[e]) for e in range(nE)]
        v_bnd = [any(f_bnd[f] for f in self.v_faces[v]) for v in range(nv)]
        self.flag_v = [boundary_flag if b else inner_flag for b in v_bnd]
        self.flag_e = [boundary_flag if b else inner_flag for b in e_bnd]
        self.flag_f = [boundary_flag if b else inner_flag for b in f_bnd]
        self.flag_c = [inner_flag] * nC
        # BoundaryCondition::create0123BC: flag 0 Inner, 1 Dirichlet, 2 Neumann, 3 Freeslip
        self.bc_types = bc_types or {0: INNER, 1: DIRICHLET, 2: NEUMANN, 3: FREESLIP}

    def bc(self, kind, idx):
        flag = {"v": self.flag_v, "e": self.flag_e, "f": self.flag_f, "c": self.flag_c}[kind][idx]
        return self.bc_types.get(flag, INNER)


# ---------------------------------------------------------------------------------------------
# meshes used by the tests and the configs
# ---------------------------------------------------------------------------------------------

def mesh_cuboid(lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), nx=1, ny=1, nz=1):
    """MeshInfo::meshCuboid (src/hyteg/mesh/MeshGenCuboid.cpp:35-172): six tets per sub-cube."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    hx, hy, hz = (x1 - x0) / nx, (y1 - y0) / ny, (z1 - z0) / nz
    coords = []
    for iz in range(nz + 1):
        for iy in range(ny + 1):
            for ix in range(nx + 1):
                coords.append((x0 + ix * hx, y0 + iy * hy, z0 + iz * hz))
    corner = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    split = [(4, 5, 7, 3), (0, 3, 1, 4), (4, 1, 5, 3), (5, 6, 7, 2), (1, 3, 2, 5), (7, 2, 3, 5)]
    tets = []
    for iz in range(nz):
        for iy in range(ny):
            for ix in range(nx):
                for t in split:
                    ids = []
                    for m in t:
                        ox, oy, oz = corner[m]
                        ids.append((iz + oz) * (nx + 1) * (ny + 1) + (iy + oy) * (nx + 1) + (ix + ox))
                    tets.append(ids)
    return np.array(coords), tets


# ---------------------------------------------------------------------------------------------
# layout of one level
# ---------------------------------------------------------------------------------------------

class Level:
    """HyTeG vertex-DoF layout of all primitives at one level, plus owner maps."""

    def __init__(self, mesh: MacroMesh, L: int):
        self.mesh, self.L = mesh, L
        n = 1 << L
        self.n = n
        m = mesh
        sizes_v = [1 + len(m.v_edges[v]) for v in range(m.nV)]
        sizes_e = [(n + 1) + len(m.e_faces[e]) * n + len(m.e_cells[e]) * (n - 1) for e in range(m.nE)]
        sizes_f = [tri_size(n + 1) + len(m.f_cells[f]) * tri_size(n) for f in range(m.nF)]
        sizes_c = [tet_size(n + 1)] * m.nC
        allsizes = sizes_v + sizes_e + sizes_f + sizes_c
        offs = np.concatenate([[0], np.cumsum(allsizes)]).astype(np.int64)
        self.size = int(offs[-1])
        self.off_v = offs[: m.nV]
        self.off_e = offs[m.nV: m.nV + m.nE]
        self.off_f = offs[m.nV + m.nE: m.nV + m.nE + m.nF]
        self.off_c = offs[m.nV + m.nE + m.nF: m.nV + m.nE + m.nF + m.nC]
        self.sizes = dict(v=sizes_v, e=sizes_e, f=sizes_f, c=sizes_c)
        self._build_owned()
        self._cell_pts = tet_points(n + 1)  # all points of a cell array in memory order

    # owned slots -----------------------------------------------------------------------------
    def _build_owned(self):
        m, n = self.mesh, self.n
        owned, bc = [], []
        for v in range(m.nV):
            owned.append(np.array([self.off_v[v]]))
            bc.append(np.full(1, m.bc("v", v)))
        for e in range(m.nE):
            idx = self.off_e[e] + np.arange(1, n)
            owned.append(idx)
            bc.append(np.full(idx.size, m.bc("e", e)))
        for f in range(m.nF):
            ij = [(i, j) for j in range(1, n) for i in range(1, n - j)]
            idx = np.array([self.off_f[f] + face_index(n, i, j) for i, j in ij], dtype=np.int64)
            owned.append(idx)
            bc.append(np.full(idx.size, m.bc("f", f)))
        for c in range(m.nC):
            pts = tet_points(n + 1)
            inner = (pts.min(axis=1) >= 1) & (pts.sum(axis=1) <= n - 1)
            idx = self.off_c[c] + cell_index(n, pts[inner, 0], pts[inner, 1], pts[inner, 2])
            owned.append(idx)
            bc.append(np.full(idx.size, m.bc("c", c)))
        self.owned = np.concatenate(owned).astype(np.int64)
        self.owned_bc = np.concatenate(bc).astype(np.int64)
        self.bc_of_slot = np.zeros(self.size, dtype=np.int64)
        self.bc_of_slot[self.owned] = self.owned_bc

    def owned_mask(self, flag=ALL):
        mask = np.zeros(self.size, dtype=bool)
        sel = (self.owned_bc & flag) != 0
        mask[self.owned[sel]] = True
        return mask

    # owner of cell-local points --------------------------------------------------------------
    def owner(self, c, x, y, z):
        """Owner slot of the cell-local micro-vertex (x, y, z) of macro-cell c (vectorised).

        The owner follows from the barycentric integer weights (n-x-y-z, x, y, z) on the
        cell's vertices: one non-zero weight -> macro-vertex, two -> macro-edge (local index =
        weight of the edge's second vertex), three -> macro-face (local (i, j) = weights of the
        face's second and third vertex), four -> cell interior.
        """
        m, n = self.mesh, self.n
        x, y, z = (np.asarray(a, dtype=np.int64) for a in (x, y, z))
        w = np.stack([n - x - y - z, x, y, z], axis=-1)
        cv = m.cells[c]
        nz = w != 0
        out = np.full(x.shape, -1, dtype=np.int64)
        patterns = {}
        key = nz[..., 0] * 1 + nz[..., 1] * 2 + nz[..., 2] * 4 + nz[..., 3] * 8
        for k in np.unique(key):
            sel = key == k
            locs = [i for i in range(4) if (k >> i) & 1]
            gv = [cv[i] for i in locs]
            if len(locs) == 1:
                out[sel] = self.off_v[gv[0]]
            elif len(locs) == 2:
                e = m.edge_id[tuple(sorted(gv))]
                ev1 = m.edges[e][1]
                wi = w[sel][:, locs[gv.index(ev1)]]
                out[sel] = self.off_e[e] + wi
            elif len(locs) == 3:
                f = m.face_id[tuple(sorted(gv))]
                fv = m.faces[f]
                wi = w[sel][:, locs[gv.index(fv[1])]]
                wj = w[sel][:, locs[gv.index(fv[2])]]
                out[sel] = self.off_f[f] + face_index(n, wi, wj)
            else:
                out[sel] = self.off_c[c] + cell_index(n, x[sel], y[sel], z[sel])
        return out

    def coords(self, c, x, y, z):
        """vertexdof::macrocell::coordinateFromIndex (VertexDoFMacroCell.hpp:70-77)."""
        cv = self.mesh.cells[c]
        P = self.mesh.vcoords[list(cv)]
        step = 1.0 / self.n
        xs, ys, zs = (P[1] - P[0]) * step, (P[2] - P[0]) * step, (P[3] - P[0]) * step
        x, y, z = (np.asarray(a, dtype=np.float64)[..., None] for a in (x, y, z))
        return P[0] + xs * x + ys * y + zs * z

    def copy_map(self):
        """(dst, src) pairs: every cell-array slot that is a copy of a lower-dimensional owner."""
        dsts, srcs = [], []
        pts = self._cell_pts
        for c in range(self.mesh.nC):
            own = self.owner(c, pts[:, 0], pts[:, 1], pts[:, 2])
            slot = self.off_c[c] + cell_index(self.n, pts[:, 0], pts[:, 1], pts[:, 2])
            sel = own != slot
            dsts.append(slot[sel])
            srcs.append(own[sel])
        return np.concatenate(dsts), np.concatenate(srcs)

    def sync(self, vec):
        """Fill cell-array copy slots from their owners (communicate<Vertex..Face, Cell>)."""
        if not hasattr(self, "_cmap"):
            self._cmap = self.copy_map()
        d, s = self._cmap
        vec[d] = vec[s]
        return vec

    def micro_cells(self, c):
        """Owner slots (k, 4) and coordinates (k, 4, 3) of all micro-cells of macro-cell c."""
        n = self.n
        slots, xyz = [], []
        for _, offs, shift in MICRO_CELL_TYPES:
            w = n - shift
            if w <= 0:
                continue
            base = tet_points(w)
            vs = [base + np.array(o, dtype=np.int64) for o in offs]
            slots.append(np.stack([self.owner(c, v[:, 0], v[:, 1], v[:, 2]) for v in vs], axis=1))
            xyz.append(np.stack([self.coords(c, v[:, 0], v[:, 1], v[:, 2]) for v in vs], axis=1))
        return np.concatenate(slots), np.concatenate(xyz)


# ---------------------------------------------------------------------------------------------
# element matrices and operators
# ---------------------------------------------------------------------------------------------

def p1_laplace_element(X):
    """P1 stiffness matrices for tets X (k, 4, 3): K = |det J|/6 * G G^T (p1_tet_diffusion form)."""
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)  # columns
    det = np.linalg.det(J)
    Jinv = np.linalg.inv(J)  # rows of Jinv are grad of lambda_1..3
    G = np.concatenate([-Jinv.sum(axis=1, keepdims=True), Jinv], axis=1)  # (k, 4, 3)
    return (np.abs(det) / 6.0)[:, None, None] * np.einsum("kid,kjd->kij", G, G)


def p1_mass_element(X):
    """P1 mass matrices: |det J|/120 * (1 + delta_ij)."""
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)
    det = np.abs(np.linalg.det(J))
    M = (np.ones((4, 4)) + np.eye(4)) / 120.0
    return det[:, None, None] * M[None]


def assemble(level: Level, element=p1_laplace_element):
    """Global matrix over HyTeG layout slots from micro-cell element matrices."""
    rows, cols, vals = [], [], []
    for c in range(level.mesh.nC):
        slots, X = level.micro_cells(c)
        K = element(X)
        rows.append(np.repeat(slots, 4, axis=1).ravel())
        cols.append(np.tile(slots, (1, 4)).ravel())
        vals.append(K.reshape(K.shape[0], 16).ravel())
    A = sp.coo_matrix(
        (np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(level.size, level.size)
    ).tocsr()
    A.sum_duplicates()
    return A


class P1ConstantLaplace:
    """P1 Laplace operator over levels minL..maxL (apply / smooth_jac / inverse diagonal)."""

    def __init__(self, mesh, minL, maxL, element=p1_laplace_element):
        self.mesh, self.minL, self.maxL = mesh, minL, maxL
        self.levels = {L: Level(mesh, L) for L in range(minL, maxL + 1)}
        self.A = {L: assemble(self.levels[L], element) for L in range(minL, maxL + 1)}
        self.invdiag = {}
        for L, A in self.A.items():
            d = A.diagonal()
            inv = np.zeros_like(d)
            own = self.levels[L].owned
            inv[own] = 1.0 / d[own]
            self.invdiag[L] = inv

    def apply(self, src, dst, L, flag, add=False):
        """P1Operator::apply: dst = A src (or dst += A src) on owned DoFs matching flag."""
        y = self.A[L] @ src
        mask = self.levels[L].owned_mask(flag)
        if add:
            dst[mask] += y[mask]
        else:
            dst[mask] = y[mask]
        return dst

    def smooth_jac(self, dst, rhs, src, relax, L, flag):
        """P1Operator::smooth_jac (P1Operator.hpp:429-447): dst = src + relax * D^-1 (rhs - A src)."""
        mask = self.levels[L].owned_mask(flag)
        y = self.A[L] @ src
        t = rhs - y
        t = self.invdiag[L] * t
        dst[mask] = src[mask] + relax * t[mask]
        return dst


# ---------------------------------------------------------------------------------------------
# grid transfer
# ---------------------------------------------------------------------------------------------

def _num_neighbor_cells_of_owner(level: Level):
    """For every slot: number of macro-cells around the owning primitive (1 for cell interior)."""
    m = level.mesh
    cnt = np.ones(level.size)
    for v in range(m.nV):
        cnt[level.off_v[v]: level.off_v[v] + level.sizes["v"][v]] = len(m.v_cells[v])
    for e in range(m.nE):
        cnt[level.off_e[e]: level.off_e[e] + level.sizes["e"][e]] = len(m.e_cells[e])
    for f in range(m.nF):
        cnt[level.off_f[f]: level.off_f[f] + level.sizes["f"][f]] = len(m.f_cells[f])
    return cnt


def restriction_matrix(fine: Level, coarse: Level):
    """restrict3D with the generated pull kernel as a matrix over owner slots.

    ``restrict_3D_macrocell_P1_pull_additive`` (gridtransferoperators/generatedKernels,
    :53-120 for the vertex-0 case) pulls, per macro-cell, the fine centre with weight 1 and the
    fine stencil neighbours with weight 1/2, each scaled by 1/(number of macro-cells around the
    primitive that owns the *fine* point); ``communicateAdditively<Cell, *>``
    (P1toP1LinearRestriction.cpp:342-344) then sums the cell shares into flagged owners.
    """
    assert fine.L == coarse.L + 1
    nc = coarse.n
    pts = tet_points(nc + 1)
    ncells = _num_neighbor_cells_of_owner(fine)
    rows, cols, vals = [], [], []
    for c in range(fine.mesh.nC):
        dst = coarse.owner(c, pts[:, 0], pts[:, 1], pts[:, 2])
        src = fine.owner(c, 2 * pts[:, 0], 2 * pts[:, 1], 2 * pts[:, 2])
        rows.append(dst), cols.append(src), vals.append(1.0 / ncells[src])
        for d in STENCIL_DIRS:
            q = 2 * pts + d
            inside = (q.min(axis=1) >= 0) & (q.sum(axis=1) <= fine.n)
            s = fine.owner(c, q[inside, 0], q[inside, 1], q[inside, 2])
            rows.append(dst[inside]), cols.append(s), vals.append(0.5 / ncells[s])
    R = sp.coo_matrix(
        (np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(coarse.size, fine.size)
    ).tocsr()
    R.sum_duplicates()
    return R


def prolongation_matrix(coarse: Level, fine: Level):
    """Linear interpolation (prolongate3DAdditively, P1toP1LinearProlongation.cpp:194-410)."""
    assert fine.L == coarse.L + 1
    pts = tet_points(fine.n + 1)
    seen = np.zeros(fine.size, dtype=bool)
    rows, cols, vals = [], [], []
    for c in range(fine.mesh.nC):
        dst = fine.owner(c, pts[:, 0], pts[:, 1], pts[:, 2])
        odd = pts % 2
        even = odd.sum(axis=1) == 0
        # the coarse micro-edge through an odd fine point has direction d in the stencil
        # set with |d_k| = odd_k; choose the representative with d_x >= 0 and d = sign pattern
        d = np.zeros_like(pts)
        for dirv in STENCIL_DIRS:
            match = np.all(np.abs(dirv)[None, :] == odd, axis=1)
            d[match] = dirv
        a = (pts - d) // 2
        b = (pts + d) // 2
        new = ~seen[dst]
        # mark first occurrence only (all cells give the same interpolation)
        uniq_dst, first = np.unique(dst[new], return_index=True)
        sel = np.flatnonzero(new)[first]
        seen[uniq_dst] = True
        ev = even[sel]
        ca = coarse.owner(c, a[sel, 0], a[sel, 1], a[sel, 2])
        cb = coarse.owner(c, b[sel, 0], b[sel, 1], b[sel, 2])
        rows.append(dst[sel][ev]), cols.append(ca[ev]), vals.append(np.ones(ev.sum()))
        ne = ~ev
        rows.append(dst[sel][ne]), cols.append(ca[ne]), vals.append(np.full(ne.sum(), 0.5))
        rows.append(dst[sel][ne]), cols.append(cb[ne]), vals.append(np.full(ne.sum(), 0.5))
    P = sp.coo_matrix(
        (np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(fine.size, coarse.size)
    ).tocsr()
    P.sum_duplicates()
    return P


class Transfer:
    def __init__(self, op: P1ConstantLaplace):
        self.op = op
        self.R, self.P = {}, {}
        for L in range(op.minL + 1, op.maxL + 1):
            self.R[L] = restriction_matrix(op.levels[L], op.levels[L - 1])
            self.P[L] = prolongation_matrix(op.levels[L - 1], op.levels[L])

    def restrict(self, fine_vec, coarse_vec, L, flag):
        """coarse (level L-1) <- R fine (level L) on flagged owned coarse DoFs."""
        y = self.R[L] @ fine_vec
        mask = self.op.levels[L - 1].owned_mask(flag)
        coarse_vec[mask] = y[mask]
        return coarse_vec

    def prolongate(self, coarse_vec, fine_vec, L, flag, add=True):
        """fine (level L) (+)= P coarse (level L-1) on flagged owned fine DoFs."""
        y = self.P[L] @ coarse_vec
        mask = self.op.levels[L].owned_mask(flag)
        if add:
            fine_vec[mask] += y[mask]
        else:
            fine_vec[mask] = y[mask]
        return fine_vec


# ---------------------------------------------------------------------------------------------
# solvers
# ---------------------------------------------------------------------------------------------

def dot(level: Level, a, b, flag):
    """dotGlobal over owned DoFs of the flagged types (VertexDoFFunction.cpp:1710-1790)."""
    mask = level.owned_mask(flag)
    return float(np.dot(a[mask], b[mask]))


def chebyshev_coefficients(order, lower, upper):
    """Coefficients c_0..c_{k-1} with x += sum_i c_i (D^-1 A)^i D^-1 r.

    Equivalent to ChebyshevSmoother::setupCoefficientsInternal (ChebyshevSmoother.hpp:329-555):
    the error polynomial 1 - t p(t) equals T_k((theta - t)/delta) / T_k(theta/delta),
    theta = (upper+lower)/2, delta = (upper-lower)/2.  Derived here by polynomial algebra.
    """
    theta = 0.5 * (upper + lower)
    delta = 0.5 * (upper - lower)
    # Chebyshev T_k as coefficient lists in s
    T = [np.array([1.0]), np.array([0.0, 1.0])]
    for k in range(2, order + 1):
        T.append(np.concatenate([[0.0], 2 * T[-1]]) - np.concatenate([T[-2], [0.0, 0.0]]))
    Tk = T[order]
    # substitute s = (theta - t)/delta  -> polynomial in t
    poly_t = np.zeros(order + 1)
    base = np.array([theta / delta, -1.0 / delta])
    powk = np.array([1.0])
    for k in range(order + 1):
        poly_t[: powk.size] += Tk[k] * powk
        powk = np.convolve(powk, base)
    norm = np.polyval(Tk[::-1], theta / delta)
    e = poly_t / norm  # e(0) = 1
    # 1 - t p(t) = e(t)  =>  p_i = -e_{i+1}
    return [-e[i + 1] for i in range(order)]


class GMG:
    """GeometricMultigridSolver (V/W cycle) with weighted Jacobi or Chebyshev smoothing."""

    def __init__(self, op, transfer, minL, maxL, pre=2, post=2, increment=0, cycle="V",
                 smoother="jacobi", omega=2.0 / 3.0, cheb_order=3, cheb_radii=None,
                 cg_tol=1e-14, cg_abs=1e-16, cg_maxit=10**6):
        self.op, self.tr = op, transfer
        self.minL, self.maxL = minL, maxL
        self.pre, self.post, self.inc, self.cycle = pre, post, increment, cycle
        self.smoother, self.omega = smoother, omega
        self.flag = INNER | NEUMANN | FREESLIP
        self.cg_tol, self.cg_abs, self.cg_maxit = cg_tol, cg_abs, cg_maxit
        if smoother == "chebyshev":
            self.cheb = {L: chebyshev_coefficients(cheb_order, 0.3 * cheb_radii[L], 1.2 * cheb_radii[L])
                         for L in range(minL, maxL + 1)}

    # smoothers -----------------------------------------------------------------------------
    def smooth(self, x, b, L):
        op = self.op
        if self.smoother == "jacobi":
            tmp = x.copy()  # tmp.assign({1}, {x}, level, All)
            op.smooth_jac(x, b, tmp, self.omega, L, self.flag)
        else:
            self.chebyshev_step(x, b, L)

    def chebyshev_step(self, x, b, L):
        """ChebyshevSmoother::solve (ChebyshevSmoother.hpp:112-240)."""
        op, lev = self.op, self.op.levels[L]
        mask = lev.owned_mask(self.flag)
        coeff = self.cheb[L]
        # copyBCs(x, tmp1/tmp2): boundary entries of the temporaries carry x's boundary values
        tmp1 = x.copy()
        tmp2 = x.copy()
        op.apply(x, tmp2, L, self.flag)
        tmp2[mask] = b[mask] - tmp2[mask]
        tmp1[mask] = op.invdiag[L][mask] * tmp2[mask]
        x[mask] = x[mask] + coeff[0] * tmp1[mask]
        for k in range(1, len(coeff)):
            op.apply(tmp1, tmp2, L, self.flag)
            tmp1[mask] = op.invdiag[L][mask] * tmp2[mask]
            x[mask] = x[mask] + coeff[k] * tmp1[mask]

    # coarse solver -------------------------------------------------------------------------
    def cg(self, x, b, L):
        """CGSolver::solve (CGSolver.hpp:94-206) with identity preconditioner."""
        op, lev, flag = self.op, self.op.levels[L], self.flag
        mask = lev.owned_mask(flag)
        r = np.zeros_like(x)
        ap = np.zeros_like(x)
        # init: r = b - A x ; p = z = r
        op.apply(x, ap, L, flag)
        r[mask] = b[mask] - ap[mask]
        p = np.where(mask, r, 0.0)
        prsold = dot(lev, r, r, flag)
        res_start = math.sqrt(prsold)
        if res_start < self.cg_abs:
            return 0
        for it in range(self.cg_maxit):
            op.apply(p, ap, L, flag)
            pAp = dot(lev, p, ap, flag)
            alpha = prsold / pAp
            x[mask] += alpha * p[mask]
            r[mask] -= alpha * ap[mask]
            rsnew = dot(lev, r, r, flag)
            sq = math.sqrt(rsnew)
            if sq / res_start < self.cg_tol or sq < self.cg_abs:
                return it
            beta = rsnew / prsold
            p[mask] = r[mask] + beta * p[mask]
            prsold = rsnew
        return self.cg_maxit

    # cycle -----------------------------------------------------------------------------------
    def solve(self, x, b, L):
        """x, b: dicts level -> layout vector.  One multigrid cycle on level L."""
        self.invoked = L
        self._rec(x, b, L)

    def _rec(self, x, b, L):
        op = self.op
        if L == self.minL:
            self.cg(x[L], b[L], L)
            return
        for _ in range(self.pre + self.inc * (self.invoked - L)):
            self.smooth(x[L], b[L], L)
        tmp = np.zeros(op.levels[L].size)
        op.apply(x[L], tmp, L, self.flag)
        mask = op.levels[L].owned_mask(self.flag)
        tmp[mask] = b[L][mask] - tmp[mask]
        coarse_tmp = np.zeros(op.levels[L - 1].size)
        self.tr.restrict(tmp, coarse_tmp, L, self.flag)
        cm = op.levels[L - 1].owned_mask(self.flag)
        b[L - 1][cm] = coarse_tmp[cm]
        x[L - 1][:] = 0.0
        self._rec(x, b, L - 1)
        if self.cycle == "W":
            self._rec(x, b, L - 1)
        self.tr.prolongate(x[L - 1], x[L], L, self.flag, add=True)
        for _ in range(self.post + self.inc * (self.invoked - L)):
            self.smooth(x[L], b[L], L)


def sor_color_sets(lev: Level):
    """Slot masks of the device Gauss-Seidel's colour sets in sweep order: macro-vertex DoFs; edge DoFs
    by the parity of their edge index; face DoFs by (i + 2j) mod 3 of their face index (i, j); cell
    interiors by (x + 2y + 3z) mod 4 of their cell-local coordinates."""
    m, n = lev.mesh, lev.n
    sets = []
    V = np.zeros(lev.size, dtype=bool)
    V[np.asarray(lev.off_v, dtype=np.int64)] = True
    sets.append(V)
    for col in (0, 1):
        S = np.zeros(lev.size, dtype=bool)
        i = np.arange(1, n)
        for e in range(m.nE):
            S[lev.off_e[e] + i[i % 2 == col]] = True
        sets.append(S)
    ij = [(i, j) for j in range(1, n) for i in range(1, n - j)]
    for col in (0, 1, 2):
        S = np.zeros(lev.size, dtype=bool)
        sel = [face_index(n, i, j) for i, j in ij if (i + 2 * j) % 3 == col]
        for f in range(m.nF):
            if sel:
                S[lev.off_f[f] + np.array(sel, dtype=np.int64)] = True
        sets.append(S)
    pts = tet_points(n + 1)
    inner = (pts.min(axis=1) >= 1) & (pts.sum(axis=1) <= n - 1)
    p = pts[inner]
    for col in range(4):
        S = np.zeros(lev.size, dtype=bool)
        q = p[(p[:, 0] + 2 * p[:, 1] + 3 * p[:, 2]) % 4 == col]
        for c in range(m.nC):
            if len(q):
                S[lev.off_c[c] + cell_index(n, q[:, 0], q[:, 1], q[:, 2])] = True
        sets.append(S)
    return sets


def sor_sweep(op, x, b, L, relax, flag, backwards=False):
    """P1Operator::smooth_sor (P1Operator.hpp:339-420) in the device's colour-set order: for each set
    S (reversed when backwards) x_S <- x_S + relax D^-1 (b - A x)_S with the values before the set,
    copies refreshed after every set."""
    lev = op.levels[L]
    own = lev.owned_mask(flag)
    sets = sor_color_sets(lev)
    if backwards:
        sets = sets[::-1]
    x = lev.sync(x.copy())
    for S in sets:
        sel = S & own
        r = b - op.A[L] @ x
        x[sel] = x[sel] + relax * (op.invdiag[L][sel] * r[sel])
        x = lev.sync(x)
    return x


def power_iteration_radius(op: P1ConstantLaplace, L, x0, iters):
    """estimateSpectralRadiusWithPowerIteration on D^-1 A (SpectrumEstimation.hpp:56-84), flag All."""
    lev = op.levels[L]
    x = x0.copy()
    aux = np.zeros_like(x)

    def dinv_a(src, dst):
        op.apply(src, dst, L, ALL)
        m = lev.owned_mask(ALL)
        dst[m] = op.invdiag[L][m] * dst[m]

    norm = math.sqrt(dot(lev, x, x, ALL))
    x = x * (1.0 / norm)
    dinv_a(x, aux)
    radius = 0.0
    for _ in range(iters):
        norm = math.sqrt(dot(lev, aux, aux, ALL))
        x = aux * (1.0 / norm)
        dinv_a(x, aux)
        radius = dot(lev, x, aux, ALL)
    return radius


def residual_norm(op, x, b, L, flag=INNER | NEUMANN | FREESLIP):
    lev = op.levels[L]
    r = np.zeros(lev.size)
    op.apply(x, r, L, flag)
    mask = lev.owned_mask(flag)
    r[mask] = b[mask] - r[mask]
    return math.sqrt(dot(lev, r, r, flag))


# ---------------------------------------------------------------------------------------------
# constant-stencil operator on one large level, without a global matrix
# ---------------------------------------------------------------------------------------------
def _face_mask(n, x, y, z):
    """Which macro-cell faces a cell-local point lies on: bit 0 z = 0, bit 1 y = 0, bit 2 x = 0,
    bit 3 x + y + z = n."""
    return (z == 0) * 1 + (y == 0) * 2 + (x == 0) * 4 + (x + y + z == n) * 8


def _mask_point(n, mask):
    """A cell-local point on exactly the faces of `mask` (n >= 4)."""
    fixed = [bool(mask & 4), bool(mask & 2), bool(mask & 1)]  # x, y, z pinned to 0
    p = [0 if f else 1 for f in fixed]
    if mask & 8:
        free = [i for i in range(3) if not fixed[i]]
        p[free[-1]] = n - (len(free) - 1)
    return np.array(p, dtype=np.int64)


def cell_stencils_by_mask(mesh: MacroMesh, c, L, element=p1_laplace_element):
    """calculateStencilInMacroCellForm_new (P1Elements.hpp:466-529) for macro-cell c: for every face
    set `mask` a cell point can lie on, the 15 stencil weights (centre, then STENCIL_DIRS), each the
    sum of the element-matrix entries K[k, j] of the micro-cells of the cell that contain the point as
    their vertex k and the neighbour as vertex j.  The cell is affine, so all points with the same
    face set share the stencil.  Returns a (16, 15) array indexed by mask."""
    n = 1 << L
    P = mesh.vcoords[list(mesh.cells[c])]
    step = (P[1:] - P[0]) / n  # micro-vertex coordinates as VertexDoFMacroCell.hpp:70-77
    dir_index = {tuple(d): i + 1 for i, d in enumerate(STENCIL_DIRS.tolist())}
    dir_index[(0, 0, 0)] = 0
    # element matrix of each micro-cell type (translates of one another inside the affine cell)
    K = []
    for _, offs, _shift in MICRO_CELL_TYPES:
        v = np.array(offs, dtype=np.int64)
        X = P[0] + v.astype(np.float64) @ step
        K.append(element(X[None])[0])
    out = np.zeros((16, 15))
    for mask in range(16):
        if mask == 15:
            continue  # no point lies on all four faces
        p = _mask_point(n, mask)
        for t, (_, offs, shift) in enumerate(MICRO_CELL_TYPES):
            v = np.array(offs, dtype=np.int64)
            for k in range(4):
                a = p - v[k]  # anchor of the micro-cell of type t holding p as vertex k
                if a.min() < 0 or a.sum() > n - shift - 1:
                    continue
                for j in range(4):
                    out[mask, dir_index[tuple((v[j] - v[k]).tolist())]] += K[t][k, j]
    return out


class LargeLevelConstantOperator:
    """P1ConstantOperator on one level without assembling the global matrix, for levels where the
    assembled oracle does not fit (level 7 and 8 parity).

    apply: cell interiors through `interior_kernel(cell_array, L, stencil15)` (the reference's compiled
    apply_3D_macrocell_vertexdof_to_vertexdof_replace when the caller passes it; cell_stencil_apply
    otherwise); every face, edge and vertex owner is the sum over its neighbour cells of the one-sided
    stencil of its position in that cell, the decomposition of P1ConstantOperator::apply_face3D_generated
    (P1ConstantOperator.cpp:239-357) and of the edge / vertex stencils (P1Operator.hpp:1044-1108), whose
    weights are the same sums of micro-cell element-matrix entries.  Interface as P1ConstantLaplace
    (apply / smooth_jac / invdiag / levels) for one level."""

    def __init__(self, mesh, L, element=p1_laplace_element, interior_kernel=None, level=None):
        self.mesh, self.L = mesh, L
        lev = level if level is not None else Level(mesh, L)
        self.levels = {L: lev}
        n = lev.n
        self.kernel = interior_kernel or cell_stencil_apply
        self.st = [cell_stencils_by_mask(mesh, c, L, element) for c in range(mesh.nC)]
        pts = lev._cell_pts
        m = _face_mask(n, pts[:, 0], pts[:, 1], pts[:, 2])
        self._bidx = np.nonzero(m != 0)[0]  # boundary points of a cell array (memory order)
        self._bmask = m[self._bidx]
        self._iidx = np.nonzero((pts.min(axis=1) >= 1) & (pts.sum(axis=1) <= n - 1))[0]
        bp = pts[self._bidx]
        self._owners = [lev.owner(c, bp[:, 0], bp[:, 1], bp[:, 2]) for c in range(mesh.nC)]
        diag = np.zeros(lev.size)
        for c in range(mesh.nC):
            diag[lev.off_c[c] + self._iidx] = self.st[c][0, 0]
            diag += np.bincount(self._owners[c], weights=self.st[c][self._bmask, 0], minlength=lev.size)
        inv = np.zeros(lev.size)
        inv[lev.owned] = 1.0 / diag[lev.owned]
        self.invdiag = {L: inv}

    def full_apply(self, src):
        """A src on every owned slot (other slots zero).  Only owner slots of src are read, as in the
        assembled operator: the cell arrays' copy slots are refreshed from their owners first."""
        lev, n, L = self.levels[self.L], self.levels[self.L].n, self.L
        src = lev.sync(np.array(src, dtype=np.float64))
        pts = lev._cell_pts
        size_c = tet_size(n + 1)
        y = np.zeros(lev.size)
        bp = pts[self._bidx]
        for c in range(self.mesh.nC):
            cell = np.ascontiguousarray(src[lev.off_c[c]: lev.off_c[c] + size_c])
            inner = self.kernel(cell, L, self.st[c][0])
            y[lev.off_c[c] + self._iidx] = inner[self._iidx]
            acc = np.zeros(self._bidx.size)
            for mask in np.unique(self._bmask):
                sel = self._bmask == mask
                P = bp[sel]
                w = self.st[c][mask]
                part = np.zeros(P.shape[0])
                for di, d in enumerate(STENCIL15):
                    if w[di] == 0.0:
                        continue  # directions leaving the cell carry no micro-cell
                    q = P + d
                    part += w[di] * cell[cell_index(n, q[:, 0], q[:, 1], q[:, 2])]
                acc[sel] = part
            y += np.bincount(self._owners[c], weights=acc, minlength=lev.size)
        return y

    def apply(self, src, dst, L, flag, add=False):
        y = self.full_apply(src)
        mask = self.levels[L].owned_mask(flag)
        if add:
            dst[mask] += y[mask]
        else:
            dst[mask] = y[mask]
        return dst

    def smooth_jac(self, dst, rhs, src, relax, L, flag):
        mask = self.levels[L].owned_mask(flag)
        t = self.invdiag[L] * (rhs - self.full_apply(src))
        dst[mask] = src[mask] + relax * t[mask]
        return dst


# ---------------------------------------------------------------------------------------------
# single macro-cell kernels (the per-cell steps of apply / restrict / prolongate)
# ---------------------------------------------------------------------------------------------
STENCIL15 = np.concatenate([np.zeros((1, 3), dtype=np.int64), STENCIL_DIRS])


def _cell_class_weight(pts, n, nc14):
    """1/(number of macro-cells around the cell sub-primitive holding each point); nc14 = edges 0-5,
    faces 0-3, vertices 0-3 of the cell."""
    x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
    on = np.stack([z == 0, y == 0, x == 0, x + y + z == n], axis=1)  # cell faces 012, 013, 023, 123
    key = on[:, 0] * 1 + on[:, 1] * 2 + on[:, 2] * 4 + on[:, 3] * 8
    table = {0: None, 1: 6, 2: 7, 4: 8, 8: 9, 3: 0, 5: 1, 9: 2, 6: 3, 10: 4, 12: 5, 7: 10, 11: 11, 13: 12, 14: 13}
    w = np.ones(len(pts))
    for k, idx in table.items():
        if idx is not None:
            w[key == k] = 1.0 / nc14[idx]
    return w


def cell_stencil_apply(src, L, stencil15):
    """apply_3D_macrocell_vertexdof_to_vertexdof_replace: interior points get sum_d s_d src[p+d]."""
    n = 1 << L
    pts = tet_points(n + 1)
    inner = (pts.min(axis=1) >= 1) & (pts.sum(axis=1) <= n - 1)
    p = pts[inner]
    out = np.zeros_like(src)
    acc = np.zeros(len(p))
    for d, s in zip(STENCIL15, stencil15):
        q = p + d
        acc += s * src[cell_index(n, q[:, 0], q[:, 1], q[:, 2])]
    out[cell_index(n, p[:, 0], p[:, 1], p[:, 2])] = acc
    return out


def cell_restrict(fine, Lc, nc14):
    """restrict_3D_macrocell_P1_pull_additive on one cell (all coarse points)."""
    nc, nf = 1 << Lc, 2 << Lc
    cp = tet_points(nc + 1)
    fc = 2 * cp
    out = _cell_class_weight(fc, nf, nc14) * fine[cell_index(nf, fc[:, 0], fc[:, 1], fc[:, 2])]
    for d in STENCIL_DIRS:
        q = fc + d
        inside = (q.min(axis=1) >= 0) & (q.sum(axis=1) <= nf)
        qi = q[inside]
        out[inside] += 0.5 * _cell_class_weight(qi, nf, nc14) * fine[cell_index(nf, qi[:, 0], qi[:, 1], qi[:, 2])]
    return out


def cell_prolongate(coarse, Lc, nc14, fine=None):
    """prolongate_3D_macrocell_P1_push_additive on one cell: fine += w * linear interpolation."""
    nc, nf = 1 << Lc, 2 << Lc
    fp = tet_points(nf + 1)
    out = np.zeros(tet_size(nf + 1)) if fine is None else fine.copy()
    odd = fp % 2
    d = np.zeros_like(fp)
    for dirv in STENCIL_DIRS:
        d[np.all(np.abs(dirv)[None, :] == odd, axis=1)] = dirv
    a, b = (fp - d) // 2, (fp + d) // 2
    ev = odd.sum(axis=1) == 0
    val = np.where(ev, coarse[cell_index(nc, a[:, 0], a[:, 1], a[:, 2])],
                   0.5 * coarse[cell_index(nc, a[:, 0], a[:, 1], a[:, 2])] + 0.5 * coarse[cell_index(nc, b[:, 0], b[:, 1], b[:, 2])])
    out[cell_index(nf, fp[:, 0], fp[:, 1], fp[:, 2])] += _cell_class_weight(fp, nf, nc14) * val
    return out


# ---------------------------------------------------------------------------------------------
# spherical shell (MeshGenSphericalShell.cpp, SHELLMESH_CLASSIC)
# ---------------------------------------------------------------------------------------------
def mesh_spherical_shell(ntan, nrad, rmin, rmax):
    """meshSphericalShell(ntan, nrad, rmin, rmax): layers equidistant in radius
    (MeshGenSphericalShell.cpp:642-660), icosahedral diamonds refined by great-circle midpoints
    (setupCoordsClassic, :420-560), vertices numbered poles first (vertIdx2Tuple / tuple2VertIdx,
    :76-195) and every local cell split into six tetrahedra with hemisphere-specific tables
    (:581-640, getCell :326-380)."""
    assert nrad >= 2 and 0 < rmin < rmax
    layers = [rmin + ((rmax - rmin) / (nrad - 1)) * k for k in range(nrad)]
    nt = ntan
    assert nt >= 2 and ((nt - 1) & (nt - 2)) == 0
    fifthpi = 0.4 * math.asin(1.0)
    w = 2.0 * math.acos(1.0 / (2.0 * math.sin(fifthpi)))
    ico = np.zeros((12, 3))
    ico[0] = (0, 0, 1.0)
    ico[11] = (0, 0, -1.0)
    for k in range(1, 6):
        phi = 2.0 * (k - 0.5) * fifthpi
        ico[k] = (math.sin(w) * math.cos(phi), math.sin(w) * math.sin(phi), math.cos(w))
        phl = 2.0 * (k - 1) * fifthpi
        ico[k + 5] = (math.sin(w) * math.cos(phl), math.sin(w) * math.sin(phl), -math.cos(w))
    dia = [(0, 5, 6, 1), (0, 1, 7, 2), (0, 2, 8, 3), (0, 3, 9, 4), (0, 4, 10, 5),
           (11, 7, 1, 6), (11, 8, 2, 7), (11, 9, 3, 8), (11, 10, 4, 9), (11, 6, 5, 10)]
    N = np.zeros((nt, nt, 10, 3))

    def mid(a, b):
        s = a + b
        return s / math.sqrt(float(s @ s))

    for d in range(10):
        L_, R_ = (1, 3) if d < 5 else (3, 1)
        N[0, 0, d] = ico[dia[d][0]]
        N[nt - 1, 0, d] = ico[dia[d][L_]]
        N[nt - 1, nt - 1, d] = ico[dia[d][2]]
        N[0, nt - 1, d] = ico[dia[d][R_]]
        m = 1
        while m < nt - 1:
            l = (nt - 1) // m
            l2 = l // 2
            for j1 in range(m + 1):
                for j2 in range(m):
                    i1, i2 = j1 * l, j2 * l + l2
                    N[i1, i2, d] = mid(N[i1, i2 - l2, d], N[i1, i2 + l2, d])
            for j1 in range(m + 1):
                for j2 in range(m):
                    i1, i2 = j2 * l + l2, j1 * l
                    N[i1, i2, d] = mid(N[i1 - l2, i2, d], N[i1 + l2, i2, d])
            for j1 in range(m):
                for j2 in range(m):
                    i1, i2 = j1 * l + l2, j2 * l + l2
                    N[i1, i2, d] = mid(N[i1 - l2, i2 + l2, d], N[i1 + l2, i2 - l2, d])
            m *= 2
    nv = (10 * (nt - 1) ** 2 + 2) * nrad
    coords = np.zeros((nv, 3))
    for v in range(nv):
        if v >= 2 * nrad:
            idx = v - 2 * nrad
            ir, idx = divmod(idx, 10 * (nt - 1) ** 2)
            d, idx = divmod(idx, (nt - 1) ** 2)
            is2, is1 = divmod(idx, nt - 1)
            is2 += 1
        elif v < nrad:
            is1, is2, d, ir = 0, 0, 0, v
        else:
            is1, is2, d, ir = 0, 0, 5, v - nrad
        coords[v] = N[is1, is2, d] * layers[ir]

    def vidx(is1, is2, d, ir):
        if is1 == 0 and is2 == 0:
            return ir if d < 5 else nrad + ir
        if is2 == 0:
            is1, is2 = 0, is1
            d = (d + 4) % 5 if d < 5 else (d + 4) % 5 + 5
        elif is1 == nt - 1:
            is1, is2 = (nt - 1) - is2, nt - 1
            d = (d + 4) % 5 + 5 if d < 5 else d % 5
        return ir * (nt - 1) ** 2 * 10 + d * (nt - 1) ** 2 + (is2 - 1) * (nt - 1) + is1 + 2 * nrad

    off = [(0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1), (0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)]
    north = [(0, 1, 3, 7), (4, 7, 5, 0), (0, 5, 1, 7), (1, 2, 3, 6), (5, 7, 6, 1), (3, 6, 7, 1)]
    south = [(4, 7, 5, 1), (0, 1, 3, 4), (4, 3, 7, 1), (7, 6, 5, 2), (3, 1, 2, 7), (5, 2, 1, 7)]
    tets = []
    for e in range((nt - 1) ** 2 * (nrad - 1) * 60):
        idx = e
        ir, idx = divmod(idx, 60 * (nt - 1) ** 2)
        d, idx = divmod(idx, 6 * (nt - 1) ** 2)
        is2, idx = divmod(idx, 6 * (nt - 1))
        is1, it = divmod(idx, 6)
        vk = []
        for o in off:
            ks1 = is1 + (o[0] if d <= 4 else o[1])
            ks2 = is2 + (o[1] if d <= 4 else o[0])
            vk.append(vidx(ks1, ks2, d, ir + o[2]))
        tab = north if d <= 4 else south
        tets.append(tuple(vk[t] for t in tab[it]))
    return coords, tets


# ---------------------------------------------------------------------------------------------
# variable-coefficient diffusion with blending (p1_div_k_grad_blending_q3)
# ---------------------------------------------------------------------------------------------
# Yu's 5-point degree-3 rule on the reference tetrahedron (volume 1/6): centroid weight -2/15,
# four points with barycentric weights (1/2, 1/6, 1/6, 1/6) and weight 3/40 each.
YU5_POINTS = np.array([[0.25, 0.25, 0.25], [1 / 6, 1 / 6, 1 / 6], [0.5, 1 / 6, 1 / 6], [1 / 6, 0.5, 1 / 6],
                       [1 / 6, 1 / 6, 0.5]])
YU5_WEIGHTS = np.array([-2.0 / 15.0, 3.0 / 40.0, 3.0 / 40.0, 3.0 / 40.0, 3.0 / 40.0])
_GHAT = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


def k_expsin(amp=0.5, phase=(0.0, 0.0, 0.0)):
    """k(x) = exp(amp sin(2 pi (x+px)) cos(2 pi (y+py)) sin(2 pi (z+pz)))."""
    tp = 2.0 * math.pi

    def k(P):
        return np.exp(amp * np.sin(tp * (P[..., 0] + phase[0])) * np.cos(tp * (P[..., 1] + phase[1]))
                      * np.sin(tp * (P[..., 2] + phase[2])))
    return k


def p1_divkgrad_element(X, kfun, blend=None, rule=(YU5_POINTS, YU5_WEIGHTS)):
    """Element matrices of -div(k grad u) for P1 on tets X (m, 4, 3) given in computational
    coordinates; blend (optional) maps computational to physical space (F, DF)."""
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)
    K = np.zeros((X.shape[0], 4, 4))
    for xi, w in zip(*rule):
        Xq = X[:, 0] + np.einsum("kij,j->ki", J, xi)
        if blend is None:
            M, Fq = J, Xq
        else:
            M, Fq = np.einsum("kij,kjl->kil", blend.DF(Xq), J), blend.F(Xq)
        det = np.abs(np.linalg.det(M))
        G = np.einsum("id,kdj->kij", _GHAT, np.linalg.inv(M))
        K += (w * kfun(Fq) * det)[:, None, None] * np.einsum("kid,kjd->kij", G, G)
    return K


class TestMap:
    """Smooth non-affine blending used to pin the form: F(x) = x (1 + a x0 x1)."""

    def __init__(self, a):
        self.a = a

    def F(self, X):
        return X * (1.0 + self.a * X[:, 0] * X[:, 1])[:, None]

    def DF(self, X):
        s = 1.0 + self.a * X[:, 0] * X[:, 1]
        g = np.stack([self.a * X[:, 1], self.a * X[:, 0], np.zeros(len(X))], axis=1)
        return s[:, None, None] * np.eye(3)[None] + X[:, :, None] * g[:, None, :]


class IcosahedralShellMap:
    """Blending of a shell macro-cell (geometry/IcosahedralShellMap.hpp:109-146, classifyVertices
    :606-705): the barycentric weight of refVertex in the tet (ray, ref, thr, for) sets the radius
    between the ray and ref radii; points are projected radially."""

    def __init__(self, mesh: MacroMesh, c, tol=1e-14):
        ref, ray, thr, fo = self._classify(mesh, c, tol)
        self.ref, self.ray, self.thr, self.fo = ref, ray, thr, fo
        self.rad_ref, self.rad_ray = np.linalg.norm(ref), np.linalg.norm(ray)
        self.bxc = np.cross(thr - ray, fo - ray)
        self.volT = float((ref - ray) @ self.bxc)

    @staticmethod
    def _classify(mesh, c, tol):
        P = mesh.vcoords[list(mesh.cells[c])]
        rad = np.linalg.norm(P, axis=1)
        inner, outer = rad.min(), rad.max()
        eps = (outer - inner) * 0.001
        n_outer = int(np.sum((outer - rad) < eps))
        pair = None
        for k in range(4):
            for j in range(k + 1, 4):
                cr = np.cross(P[k], P[j])
                if np.all(np.abs(cr) / (rad[k] * rad[j]) <= tol):
                    pair = (k, j)
                    break
            if pair:
                break
        assert pair is not None, "no radial vertex pair"
        iref, iray = pair
        if n_outer == 2:  # skew: use a non-skew neighbour of the same prism
            vref, vray = mesh.cells[c][iref], mesh.cells[c][iray]
            for f in mesh.cell_faces[c]:
                fv = mesh.faces[f]
                if not (vref in fv and vray in fv):
                    other = [cc for cc in mesh.f_cells[f] if cc != c]
                    return IcosahedralShellMap._classify(mesh, other[0], tol)
            raise AssertionError("no non-skew neighbour")
        rest = [k for k in range(4) if k not in (iref, iray)]
        ithr, ifor = rest[-1], rest[0]
        if (n_outer == 1 and rad[iref] < rad[iray]) or (n_outer == 3 and rad[iref] > rad[iray]):
            iref, iray = iray, iref
        return P[iref].copy(), P[iray].copy(), P[ithr].copy(), P[ifor].copy()

    def F(self, X):
        bary = np.abs(((X - self.ray) @ self.bxc) / self.volT)
        new_rad = self.rad_ray + bary * (self.rad_ref - self.rad_ray)
        return X * (new_rad / np.linalg.norm(X, axis=1))[:, None]

    def DF(self, X):
        r = np.linalg.norm(X, axis=1)
        bary = ((X - self.ray) @ self.bxc) / self.volT
        sgn = np.sign(bary)
        R = self.rad_ray + np.abs(bary) * (self.rad_ref - self.rad_ray)
        gradR = (self.rad_ref - self.rad_ray) * (sgn[:, None] * self.bxc[None, :] / self.volT)
        s = R / r
        grads = gradR / r[:, None] - (R / r ** 3)[:, None] * X
        return s[:, None, None] * np.eye(3)[None] + X[:, :, None] * grads[:, None, :]


class P1DivKGrad(P1ConstantLaplace):
    """P1ElementwiseBlendingDivKGradOperator (elementwiseoperators/P1ElementwiseOperator.cpp) with
    p1_div_k_grad_blending_q3: assembled from micro-cell element matrices with the coefficient k and,
    for blending="shell", the IcosahedralShellMap of every macro-cell."""

    def __init__(self, mesh, minL, maxL, kfun, blending=None):
        self.mesh, self.minL, self.maxL = mesh, minL, maxL
        self.maps = [IcosahedralShellMap(mesh, c) for c in range(mesh.nC)] if blending == "shell" else None
        self.levels = {L: Level(mesh, L) for L in range(minL, maxL + 1)}
        self.A = {}
        for L in range(minL, maxL + 1):
            lev = self.levels[L]
            rows, cols, vals = [], [], []
            for c in range(mesh.nC):
                slots, X = lev.micro_cells(c)
                K = p1_divkgrad_element(X.reshape(-1, 4, 3), kfun, None if self.maps is None else _PerPointMap(self.maps[c]))
                rows.append(np.repeat(slots, 4, axis=1).ravel())
                cols.append(np.tile(slots, (1, 4)).ravel())
                vals.append(K.reshape(K.shape[0], 16).ravel())
            A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                              shape=(lev.size, lev.size)).tocsr()
            A.sum_duplicates()
            self.A[L] = A
        self.invdiag = {}
        for L, A in self.A.items():
            d = A.diagonal()
            inv = np.zeros_like(d)
            own = self.levels[L].owned
            inv[own] = 1.0 / d[own]
            self.invdiag[L] = inv


class _PerPointMap:
    def __init__(self, m):
        self.m = m

    def F(self, X):
        return self.m.F(X)

    def DF(self, X):
        return self.m.DF(X)


# ---------------------------------------------------------------------------------------------
# P2: quadratic Lagrange elements (4 vertex DoFs, 6 edge-midpoint DoFs)
# ---------------------------------------------------------------------------------------------
# Xiao-Gimbutas degree-4 rule on the tetrahedron, 11 points, given by barycentric coordinates
# (l0, l1, l2, l3); the rule the reference's p2_div_k_grad_blending_q4 form is generated with
# (forms/form_hyteg_generated/p2/p2_div_k_grad_blending_q4.hpp:95-105).  The weights are not
# transcribed: xg4_weights() derives them from exactness for all polynomials of degree <= 4.
XG4_BARY = np.array([
    [0.17469405869723054, 0.04049050672759043, 0.01356070187980288, 0.7712547326953761],
    [0.08140491840285922, 0.752508507009655, 0.06809937093820666, 0.09798720364927911],
    [0.3044484024344971, 0.2402766649280726, 0.126801725915392, 0.3284732067220384],
    [0.7412288820936226, 0.0672232948933834, 0.03518392977359872, 0.1563638932393953],
    [0.053341239535745266, 0.419266313879513, 0.04778143555908666, 0.4796110110256551],
    [0.4329534904813558, 0.4507658760912768, 0.05945661629943383, 0.05682401712793367],
    [0.5380072039161857, 0.1294113737889104, 0.3301904148374645, 0.002391007457439365],
    [0.008991260093335729, 0.1215419913339278, 0.3064939884296903, 0.5629727601430461],
    [0.10660417256199362, 0.09720464458758327, 0.68439041545304, 0.1118007673973831],
    [0.3292329597426468, 0.02956949520647961, 0.3179035602133946, 0.323293984837479],
    [0.10384411641099309, 0.4327102390477686, 0.3538232392092971, 0.1096224053319412],
])
XG4_POINTS = XG4_BARY[:, 1:].copy()  # reference coordinates (xi1, xi2, xi3) = (l1, l2, l3)


def xg4_weights(points=XG4_POINTS, degree=4):
    """Weights of a cubature on the reference tetrahedron from the moment equations
    sum_q w_q xi^a = a1! a2! a3! / (|a| + 3)! for all |a| <= degree (least squares; exact for a
    rule of that degree)."""
    rows, rhs = [], []
    for a in range(degree + 1):
        for b in range(degree + 1 - a):
            for c in range(degree + 1 - a - b):
                rows.append(points[:, 0] ** a * points[:, 1] ** b * points[:, 2] ** c)
                rhs.append(math.factorial(a) * math.factorial(b) * math.factorial(c) / math.factorial(a + b + c + 3))
    w, *_ = np.linalg.lstsq(np.array(rows), np.array(rhs), rcond=None)
    return w


XG4_WEIGHTS = xg4_weights()
# element DoFs: vertices 0..3, then the edges in this order (FEniCS ordering,
# edgedofspace/EdgeDoFIndexing.hpp getEdgeDoFDataIndicesFromMicroVerticesFEniCSOrdering)
P2_EDGES = ((2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1))
_LGRAD = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


def p2_ref_gradients(xi):
    """Gradients (10, 3) of the quadratic Lagrange basis at reference point xi."""
    lam = np.array([1.0 - xi[0] - xi[1] - xi[2], xi[0], xi[1], xi[2]])
    G = np.zeros((10, 3))
    for i in range(4):
        G[i] = (4.0 * lam[i] - 1.0) * _LGRAD[i]
    for e, (i, j) in enumerate(P2_EDGES):
        G[4 + e] = 4.0 * (lam[i] * _LGRAD[j] + lam[j] * _LGRAD[i])
    return G


def p2_divkgrad_element(X, kfun, blend=None, rule=None):
    """Element matrices (m, 10, 10) of -div(k grad u) for P2 on tets X (m, 4, 3) in computational
    coordinates, blending map optional (same structure as p1_divkgrad_element)."""
    pts, wts = rule if rule is not None else (XG4_POINTS, XG4_WEIGHTS)
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)
    K = np.zeros((X.shape[0], 10, 10))
    for xi, w in zip(pts, wts):
        Xq = X[:, 0] + np.einsum("kij,j->ki", J, xi)
        if blend is None:
            M, Fq = J, Xq
        else:
            M, Fq = np.einsum("kij,kjl->kil", blend.DF(Xq), J), blend.F(Xq)
        det = np.abs(np.linalg.det(M))
        G = np.einsum("id,kdj->kij", p2_ref_gradients(xi), np.linalg.inv(M))
        K += (w * kfun(Fq) * det)[:, None, None] * np.einsum("kid,kjd->kij", G, G)
    return K


def p2_micro_cells(lev1, c):
    """P2 elements of level L on the nodes of Level L+1 (lev1): every level-L micro-cell of macro-cell
    c with owner slots (k, 10) of its vertex and edge-midpoint nodes (element DoF order) and its
    vertex coordinates (k, 4, 3).  A P2 function on level L has exactly the node set of level L+1."""
    n = lev1.n // 2
    slots, xyz = [], []
    for _, offs, shift in MICRO_CELL_TYPES:
        w = n - shift
        if w <= 0:
            continue
        base = tet_points(w)
        V = [2 * (base + np.array(o, dtype=np.int64)) for o in offs]
        nodes = V + [(V[i] + V[j]) // 2 for i, j in P2_EDGES]
        slots.append(np.stack([lev1.owner(c, v[:, 0], v[:, 1], v[:, 2]) for v in nodes], axis=1))
        xyz.append(np.stack([lev1.coords(c, v[:, 0], v[:, 1], v[:, 2]) for v in V], axis=1))
    return np.concatenate(slots), np.concatenate(xyz)


class P2DivKGrad(P1ConstantLaplace):
    """P2ElementwiseBlendingDivKGradOperator (elementwiseoperators/P2ElementwiseOperator.cpp:109-318,
    typedef .hpp:475) with p2_div_k_grad_blending_q4, assembled from the 10x10 element matrices of every
    micro-cell.  P2 level L lives on the node set of level L+1: levels[L] is Level(mesh, L+1)."""

    def __init__(self, mesh, minL, maxL, kfun, blending=None):
        self.mesh, self.minL, self.maxL = mesh, minL, maxL
        self.maps = [IcosahedralShellMap(mesh, c) for c in range(mesh.nC)] if blending == "shell" else None
        self.levels = {L: Level(mesh, L + 1) for L in range(minL, maxL + 1)}
        self.A = {}
        for L in range(minL, maxL + 1):
            lev = self.levels[L]
            rows, cols, vals = [], [], []
            for c in range(mesh.nC):
                slots, X = p2_micro_cells(lev, c)
                K = p2_divkgrad_element(X, kfun, None if self.maps is None else _PerPointMap(self.maps[c]))
                rows.append(np.repeat(slots, 10, axis=1).ravel())
                cols.append(np.tile(slots, (1, 10)).ravel())
                vals.append(K.reshape(K.shape[0], 100).ravel())
            A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                              shape=(lev.size, lev.size)).tocsr()
            A.sum_duplicates()
            self.A[L] = A
        self.invdiag = {}
        for L, A in self.A.items():
            d = A.diagonal()
            inv = np.zeros_like(d)
            own = self.levels[L].owned
            inv[own] = 1.0 / d[own]
            self.invdiag[L] = inv


def p2_divkgrad_element_nodal(X, knodes, blend=None):
    """Element matrices (m, 10, 10) of -div(k_h grad u) where k_h is the P2 interpolant of k: knodes
    (m, 10) holds k at the element's nodes (element DoF order) and k_h at a quadrature point is
    sum_i phi_i(xi_q) knodes_i.  This is the form of the hyteg-operators P2ElementwiseDivKGrad /
    P2ElementwiseDivKGradIcosahedralShellMap (called at tests/hyteg/convergence/
    ElementwiseDivKGradCGConvergenceTest.cpp:85-92 with k interpolated into a P2Function), restated here:
    the generated operator code lives in the hyteg_operators submodule, absent from the reference tree,
    so parity with it is unpinned.  Same rule (degree-4, 11 points) and blending as p2_divkgrad_element."""
    phi = p2_basis(XG4_BARY)  # (11, 10)
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)
    K = np.zeros((X.shape[0], 10, 10))
    for q, (xi, w) in enumerate(zip(XG4_POINTS, XG4_WEIGHTS)):
        Xq = X[:, 0] + np.einsum("kij,j->ki", J, xi)
        M = J if blend is None else np.einsum("kij,kjl->kil", blend.DF(Xq), J)
        det = np.abs(np.linalg.det(M))
        G = np.einsum("id,kdj->kij", p2_ref_gradients(xi), np.linalg.inv(M))
        kq = knodes @ phi[q]
        K += (w * kq * det)[:, None, None] * np.einsum("kid,kjd->kij", G, G)
    return K


def p2_element_nodes(X):
    """Computational coordinates (m, 10, 3) of the ten nodes of P2 elements with vertices X (m, 4, 3)."""
    return np.concatenate([X, np.stack([(X[:, i] + X[:, j]) / 2 for i, j in P2_EDGES], axis=1)], axis=1)


class P2DivKGradNodal(P1ConstantLaplace):
    """-div(k_h grad u) with k_h the P2 interpolant of kfun at the (blended) nodes of each level, assembled
    from p2_divkgrad_element_nodal (levels[L] is Level(mesh, L+1), as for P2DivKGrad)."""

    def __init__(self, mesh, minL, maxL, kfun, blending=None):
        self.mesh, self.minL, self.maxL = mesh, minL, maxL
        self.maps = [IcosahedralShellMap(mesh, c) for c in range(mesh.nC)] if blending == "shell" else None
        self.levels = {L: Level(mesh, L + 1) for L in range(minL, maxL + 1)}
        self.A = {}
        for L in range(minL, maxL + 1):
            lev = self.levels[L]
            rows, cols, vals = [], [], []
            for c in range(mesh.nC):
                slots, X = p2_micro_cells(lev, c)
                nodes = p2_element_nodes(X)
                phys = nodes if self.maps is None else self.maps[c].F(nodes.reshape(-1, 3)).reshape(nodes.shape)
                knodes = kfun(phys)
                K = p2_divkgrad_element_nodal(X, knodes, None if self.maps is None else _PerPointMap(self.maps[c]))
                rows.append(np.repeat(slots, 10, axis=1).ravel())
                cols.append(np.tile(slots, (1, 10)).ravel())
                vals.append(K.reshape(K.shape[0], 100).ravel())
            A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                              shape=(lev.size, lev.size)).tocsr()
            A.sum_duplicates()
            self.A[L] = A
        self.invdiag = {}
        for L, A in self.A.items():
            d = A.diagonal()
            inv = np.zeros_like(d)
            own = self.levels[L].owned
            inv[own] = 1.0 / d[own]
            self.invdiag[L] = inv


def p2_basis(mu):
    """Quadratic Lagrange basis (k, 10) at barycentric points mu (k, 4), element DoF order."""
    out = [mu[:, i] * (2.0 * mu[:, i] - 1.0) for i in range(4)]
    out += [4.0 * mu[:, i] * mu[:, j] for i, j in P2_EDGES]
    return np.stack(out, axis=1)


def p2_prolongation_matrix(lev_c1, lev_f1):
    """Quadratic interpolation from P2 level L-1 (nodes of Level L, lev_c1) to P2 level L (nodes of
    Level L+1, lev_f1): P2toP2QuadraticProlongation (P2toP2QuadraticProlongation.cpp:217-424).
    Every fine node takes the coarse quadratic of a level-(L-1) micro-cell containing it; shared
    nodes get identical rows from every containing micro-cell (continuity), kept once."""
    nc = lev_c1.n // 2  # micro-cells per edge on coarse P2 level
    mus = tet_points(5)  # barycentric numerators (a1, a2, a3) with a0 = 4 - a1 - a2 - a3
    rows, cols, vals = [], [], []
    seen = np.zeros(lev_f1.size, dtype=bool)
    for c in range(lev_c1.mesh.nC):
        for _, offs, shift in MICRO_CELL_TYPES:
            w = nc - shift
            if w <= 0:
                continue
            base = tet_points(w)
            Vc = [2 * (base + np.array(o, dtype=np.int64)) for o in offs]  # coarse nodes in Level-L coords
            cnodes = Vc + [(Vc[i] + Vc[j]) // 2 for i, j in P2_EDGES]
            cslots = np.stack([lev_c1.owner(c, v[:, 0], v[:, 1], v[:, 2]) for v in cnodes], axis=1)
            for a in mus:
                a0 = 4 - a.sum()
                mu = np.array([a0, a[0], a[1], a[2]], dtype=float) / 4.0
                # fine node in Level-(L+1) coords: 2 * (barycentric combination of coarse vertices)
                Pf = (a0 * 2 * Vc[0] + a[0] * 2 * Vc[1] + a[1] * 2 * Vc[2] + a[2] * 2 * Vc[3]) // 4
                fs = lev_f1.owner(c, Pf[:, 0], Pf[:, 1], Pf[:, 2])
                new = ~seen[fs]
                # one row per fine owner: drop duplicates inside this batch too
                _, first = np.unique(fs, return_index=True)
                keep = np.zeros(len(fs), dtype=bool)
                keep[first] = True
                keep &= new
                if not keep.any():
                    continue
                seen[fs[keep]] = True
                N = p2_basis(mu[None])[0]
                for j in range(10):
                    if N[j] != 0.0:
                        rows.append(fs[keep])
                        cols.append(cslots[keep, j])
                        vals.append(np.full(keep.sum(), N[j]))
    return sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(lev_f1.size, lev_c1.size)).tocsr()


class P2Transfer(Transfer):
    """P2toP2QuadraticProlongation / P2toP2QuadraticRestriction as matrices: P quadratic interpolation,
    R = P^T (the reference's per-cell scaling plus additive communication sums every fine DoF once)."""

    def __init__(self, op: P2DivKGrad):
        self.op = op
        self.R, self.P = {}, {}
        for L in range(op.minL + 1, op.maxL + 1):
            self.P[L] = p2_prolongation_matrix(op.levels[L - 1], op.levels[L])
            self.R[L] = self.P[L].T.tocsr()


# ---------------------------------------------------------------------------------------------
# the reference's P2Function memory layout (VertexDoFFunction + EdgeDoFFunction of level l)
# ---------------------------------------------------------------------------------------------

def edgedof_memory_sizes(mesh: MacroMesh, L: int):
    """Per-primitive edge-DoF array sizes in the order vertices, edges, faces, cells
    (edgeDoFMacro{Vertex,Edge,Face,Cell}FunctionMemorySize, EdgeDoFFunction.cpp:1642-1690)."""
    n = 1 << L
    out = [len(mesh.v_edges[v]) + len(mesh.v_faces[v]) for v in range(mesh.nV)]
    for e in range(mesh.nE):
        nf, nc = len(mesh.e_faces[e]), len(mesh.e_cells[e])
        out.append(1 + 2 * nf + nc if L == 0 else n + nf * (3 * n - 1) + nc * (7 * n - 7))
    for f in range(mesh.nF):
        ghost = 3 * tri_size(n) + tri_size(n - 1) + 3 * tri_size(n - 1)
        out.append(3 * tri_size(n) + len(mesh.f_cells[f]) * ghost)
    out += [6 * tet_size(n) + tet_size(n - 1)] * mesh.nC
    return out


def p2_reference_dof_coords(mesh: MacroMesh, L: int):
    """Physical coordinates (k, 3) of every entry of the reference's P2 memory of level L: the
    vertex-DoF arrays (P1 layout, closure entries) then the edge-DoF arrays (own micro-edge
    midpoints: edgedof::macroedge::index, macroface::index X / XY / Y, macrocell::xIndex..xyzIndex,
    EdgeDoFIndexing.hpp:361-366,579-594,922-980).  Ghost-layer entries are NaN."""
    n = 1 << L
    lev = Level(mesh, L)
    X = mesh.vcoords
    vpart = np.full((lev.size, 3), np.nan)
    for v in range(mesh.nV):
        vpart[lev.off_v[v]] = X[v]
    for e, (a, b) in enumerate(mesh.edges):
        t = np.arange(n + 1)[:, None] / n
        vpart[lev.off_e[e] + np.arange(n + 1)] = X[a] + t * (X[b] - X[a])
    for f, (a, b, c) in enumerate(mesh.faces):
        for j in range(n + 1):
            for i in range(n + 1 - j):
                vpart[lev.off_f[f] + face_index(n, i, j)] = X[a] + i / n * (X[b] - X[a]) + j / n * (X[c] - X[a])
    for c in range(mesh.nC):
        pts = tet_points(n + 1)
        vpart[lev.off_c[c] + cell_index(n, pts[:, 0], pts[:, 1], pts[:, 2])] = lev.coords(c, pts[:, 0], pts[:, 1], pts[:, 2])
    sizes = edgedof_memory_sizes(mesh, L)
    epart = np.full((sum(sizes), 3), np.nan)
    base = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    p = mesh.nV
    for e, (a, b) in enumerate(mesh.edges):
        t = (np.arange(n)[:, None] + 0.5) / n
        epart[base[p + e] + np.arange(n)] = X[a] + t * (X[b] - X[a])
    p += mesh.nE
    ts = tri_size(n)
    for f, (a, b, c) in enumerate(mesh.faces):
        for y in range(n):
            for x in range(n - y):
                k = base[p + f] + face_index(n - 1, x, y)
                for blk, (dx, dy) in enumerate(((0.5, 0.0), (0.5, 0.5), (0.0, 0.5))):  # X, XY, Y
                    epart[k + blk * ts] = X[a] + (x + dx) / n * (X[b] - X[a]) + (y + dy) / n * (X[c] - X[a])
    p += mesh.nF
    tb = tet_size(n)
    shifts = ((0.5, 0, 0), (0, 0.5, 0), (0, 0, 0.5), (0.5, 0.5, 0), (0.5, 0, 0.5), (0, 0.5, 0.5))  # X Y Z XY XZ YZ
    for c in range(mesh.nC):
        pts = tet_points(n)
        k = base[p + c] + cell_index(n - 1, pts[:, 0], pts[:, 1], pts[:, 2])
        for blk, d in enumerate(shifts):
            q = pts + np.array(d)
            epart[k + blk * tb] = lev.coords(c, q[:, 0], q[:, 1], q[:, 2])
        if n > 1:
            pts = tet_points(n - 1)
            q = pts + 0.5
            epart[base[p + c] + 6 * tb + cell_index(n - 2, pts[:, 0], pts[:, 1], pts[:, 2])] = lev.coords(c, q[:, 0], q[:, 1], q[:, 2])
    return np.concatenate([vpart, epart])


# ---------------------------------------------------------------------------------------------
# P2-P1 Taylor-Hood Stokes (P2P1ElementwiseBlendingStokesOperator with the velocity block
# -div(eta grad) per component, UzawaSmoother block-Laplace variant, multigrid)
# ---------------------------------------------------------------------------------------------
_QA, _QB = (5.0 - 5.0 ** 0.5) / 20.0, (5.0 + 3.0 * 5.0 ** 0.5) / 20.0
Q2_POINTS = np.array([[_QA, _QA, _QA], [_QB, _QA, _QA], [_QA, _QB, _QA], [_QA, _QA, _QB]])
Q2_WEIGHT = 1.0 / 24.0  # the 4-point degree-2 rule on the reference tetrahedron (volume 1/6)


def k_radial(amp=2.99, r0=1.0, scale=0.45):
    """Radial viscosity eta(x) = exp(amp (r0 - |x|) / scale)."""
    def k(P):
        P = np.asarray(P, dtype=np.float64)
        return np.exp(amp * (r0 - np.sqrt((P * P).sum(axis=-1))) / scale)
    return k


def p2p1_div_element(X, blend=None):
    """Element matrices (m, 3, 4, 10) of the div blocks p2_to_p1_div_{0,1,2}_blending_q2
    (P2ToP1ElementwiseBlendingDiv{x,y,z}Operator): B_k[i][j] = -int psi_i d(phi_j)/dx_k, psi P1
    (micro-cell vertices), phi P2 (element DoF order), 4-point degree-2 rule; divT is the transpose."""
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)
    B = np.zeros((X.shape[0], 3, 4, 10))
    for xi in Q2_POINTS:
        Xq = X[:, 0] + np.einsum("kij,j->ki", J, xi)
        M = J if blend is None else np.einsum("kij,kjl->kil", blend.DF(Xq), J)
        det = np.abs(np.linalg.det(M))
        G = np.einsum("id,kdj->kij", p2_ref_gradients(xi), np.linalg.inv(M))  # (m, 10, 3)
        lam = np.array([1.0 - xi.sum(), xi[0], xi[1], xi[2]])
        B -= (Q2_WEIGHT * det)[:, None, None, None] * lam[None, None, :, None] * G.transpose(0, 2, 1)[:, :, None, :]
    return B


def p2_full_viscous_element(X, mufun, blend=None, rule=(YU5_POINTS, YU5_WEIGHTS)):
    """Element matrices (m, 3, 3, 10, 10) of the full viscous velocity block
    (P2ElementwiseBlendingFullViscousOperator.hpp:34-68, forms p2_full_stokesvar_{i}_{j}_blending_q3,
    Yu's 5-point degree-3 rule): block (i, j) maps component j of the trial function to component i
    of the test function, int 2 mu eps(phi_b e_j) : eps(phi_a e_i) - (2/3) mu div(phi_b e_j) div(phi_a e_i)
    = int mu (delta_ij grad phi_a . grad phi_b + d_j phi_a d_i phi_b - (2/3) d_i phi_a d_j phi_b),
    with mu evaluated at the blended quadrature point."""
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)
    K = np.zeros((X.shape[0], 3, 3, 10, 10))
    eye = np.eye(3)
    for xi, w in zip(*rule):
        Xq = X[:, 0] + np.einsum("kij,j->ki", J, xi)
        if blend is None:
            M, Fq = J, Xq
        else:
            M, Fq = np.einsum("kij,kjl->kil", blend.DF(Xq), J), blend.F(Xq)
        s = w * mufun(Fq) * np.abs(np.linalg.det(M))
        G = np.einsum("id,kdj->kij", p2_ref_gradients(xi), np.linalg.inv(M))  # (m, 10, 3)
        lap = np.einsum("kad,kbd->kab", G, G)
        K += s[:, None, None, None, None] * (
            eye[None, :, :, None, None] * lap[:, None, None]
            + np.einsum("kaj,kbi->kijab", G, G)
            - (2.0 / 3.0) * np.einsum("kai,kbj->kijab", G, G))
    return K


def p1_pspg_element(X):
    """Element matrices (m, 4, 4) of the P1 PSPG form (p1_tet_pspg_tet.h) on affine tets:
    -(|T|^(2/3) / 12) |T| grad l_i . grad l_j."""
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)
    Ji = np.linalg.inv(J)
    G = np.concatenate([-Ji.sum(axis=1, keepdims=True), Ji], axis=1)  # rows: gradients of l_0..l_3
    vol = np.abs(np.linalg.det(J)) / 6.0
    return (-(vol ** (2.0 / 3.0)) / 12.0 * vol)[:, None, None] * np.einsum("kid,kjd->kij", G, G)


class P2FullViscous:
    """P2ElementwiseBlendingFullViscousOperator (elementwiseoperators/P2ElementwiseBlendingFullViscousOperator
    .hpp:34-68): the 3 x 3 block operator of p2_full_stokesvar_{i}_{j}_blending_q3 assembled from the
    element matrices of every micro-cell; apply follows VectorToVectorOperator::apply (dst_i = sum_j
    A_ij src_j on the flagged owned DoFs).  P2 level L lives on the node set of Level L+1."""

    def __init__(self, mesh, minL, maxL, mufun, blending=None):
        self.mesh, self.minL, self.maxL = mesh, minL, maxL
        self.maps = [IcosahedralShellMap(mesh, c) for c in range(mesh.nC)] if blending == "shell" else None
        self.levels = {L: Level(mesh, L + 1) for L in range(minL, maxL + 1)}
        self.A, self.invdiag = {}, {}
        for L in range(minL, maxL + 1):
            lev = self.levels[L]
            rows, cols, vals = [], [], [[[] for _ in range(3)] for _ in range(3)]
            for c in range(mesh.nC):
                slots, X = p2_micro_cells(lev, c)
                K = p2_full_viscous_element(X, mufun, None if self.maps is None else _PerPointMap(self.maps[c]))
                rows.append(np.repeat(slots, 10, axis=1).ravel())
                cols.append(np.tile(slots, (1, 10)).ravel())
                for i in range(3):
                    for j in range(3):
                        vals[i][j].append(K[:, i, j].reshape(K.shape[0], 100).ravel())
            r, cc = np.concatenate(rows), np.concatenate(cols)
            self.A[L] = [[sp.coo_matrix((np.concatenate(vals[i][j]), (r, cc)), shape=(lev.size, lev.size)).tocsr()
                          for j in range(3)] for i in range(3)]
            own = lev.owned
            inv = []
            for i in range(3):
                d = self.A[L][i][i].diagonal()
                v = np.zeros_like(d)
                v[own] = 1.0 / d[own]
                inv.append(v)
            self.invdiag[L] = inv

    def apply(self, src, dst, L, flag, add=False):
        mask = self.levels[L].owned_mask(flag)
        for i in range(3):
            y = sum(self.A[L][i][j] @ src[j] for j in range(3))
            if add:
                dst[i][mask] += y[mask]
            else:
                dst[i][mask] = y[mask]
        return dst


def p1_lumped_mass_inv_k_diag(X, kfun, blend=None):
    """(m, 4): minus the lumped P1 mass matrix weighted by 1/k on micro-cells X (m, 4, 3), i.e.
    -int l_i / k over the (blended) cell with Yu's 5-point rule: the viscosity-weighted pressure mass
    (the P1LumpedInvMassOperator pattern of P2P1Stokes3DUzawaConvergenceTest.cpp:125-139 with the 1/eta
    weight a variable viscosity puts into the Schur complement), negative like the PSPG diagonal."""
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)
    out = np.zeros((X.shape[0], 4))
    for xi, w in zip(YU5_POINTS, YU5_WEIGHTS):
        Xq = X[:, 0] + np.einsum("kij,j->ki", J, xi)
        if blend is None:
            M, Fq = J, Xq
        else:
            M, Fq = np.einsum("kij,kjl->kil", blend.DF(Xq), J), blend.F(Xq)
        det = np.abs(np.linalg.det(M))
        lam = np.array([1.0 - xi[0] - xi[1] - xi[2], xi[0], xi[1], xi[2]])
        out -= (w * det / kfun(Fq))[:, None] * lam[None, :]
    return out


class P2P1Stokes:
    """The Taylor-Hood system [A 0 0 B0^T; 0 A 0 B1^T; 0 0 A B2^T; B0 B1 B2 0] on P2 level L (velocity,
    nodes of Level L+1) and P1 level L (pressure), A = -div(eta grad) per component, with the
    inverted PSPG diagonal (P1PSPGInvDiagOperator, affine macro geometry) for the Uzawa step.
    Velocity rows/columns use the inner DoFs, pressure rows/columns all DoFs."""

    def __init__(self, mesh, minL, maxL, eta, blending=None, full_viscous=False, pressure_scaling="pspg"):
        self.mesh, self.minL, self.maxL = mesh, minL, maxL
        self.Aop = P2DivKGrad(mesh, minL, maxL, eta, blending)
        # the full viscous velocity block (P2ElementwiseBlendingFullViscousOperator) in place of
        # -div(eta grad) per component, smoothed by Chebyshev on the coupled block
        self.Vop = P2FullViscous(mesh, minL, maxL, eta, blending) if full_viscous else None
        self.ulev = self.Aop.levels
        self.plev = {L: Level(mesh, L) for L in range(minL, maxL + 1)}
        maps = self.Aop.maps
        self.B, self.sinv = {}, {}
        for L in range(minL, maxL + 1):
            ul, pl = self.ulev[L], self.plev[L]
            rows, cols, vals = [[], [], []], [[], [], []], [[], [], []]
            d = np.zeros(pl.size)
            for c in range(mesh.nC):
                uslots, X = p2_micro_cells(ul, c)
                # P1 owners of the micro-cell vertices: level-L coordinates are half the storage ones
                n = pl.n
                pslots = []
                for _, offs, shift in MICRO_CELL_TYPES:
                    w = n - shift
                    if w <= 0:
                        continue
                    base = tet_points(w)
                    V = [base + np.array(o, dtype=np.int64) for o in offs]
                    pslots.append(np.stack([pl.owner(c, v[:, 0], v[:, 1], v[:, 2]) for v in V], axis=1))
                pslots = np.concatenate(pslots)
                Be = p2p1_div_element(X, None if maps is None else _PerPointMap(maps[c]))
                for k in range(3):
                    rows[k].append(np.repeat(pslots, 10, axis=1).ravel())
                    cols[k].append(np.tile(uslots, (1, 4)).ravel())
                    vals[k].append(Be[:, k].reshape(-1))
                if pressure_scaling == "lumped_mass":
                    # minus the lumped pressure mass weighted by 1/eta, on the blended micro-cell
                    np.add.at(d, pslots.ravel(),
                              p1_lumped_mass_inv_k_diag(X, eta, None if maps is None else _PerPointMap(maps[c])).ravel())
                else:
                    # PSPG diagonal on the affine (computational) micro-cell
                    Kp = p1_pspg_element(X)
                    np.add.at(d, pslots.ravel(), np.einsum("kii->ki", Kp).ravel())
            self.B[L] = [sp.coo_matrix((np.concatenate(vals[k]), (np.concatenate(rows[k]), np.concatenate(cols[k]))),
                                       shape=(pl.size, ul.size)).tocsr() for k in range(3)]
            inv = np.zeros(pl.size)
            inv[pl.owned] = 1.0 / d[pl.owned]
            self.sinv[L] = inv
        self.utr = P2Transfer(self.Aop)
        self.ptr = Transfer(P1ConstantLaplace(mesh, minL, maxL))

    # --- blocks -----------------------------------------------------------------------------
    def umask(self, L):
        return self.ulev[L].owned_mask(INNER | NEUMANN | FREESLIP)

    def pmask(self, L):
        return self.plev[L].owned_mask(ALL)

    def div(self, u, L):
        """div u on all pressure DoFs (copies refreshed)."""
        r = sum(self.B[L][k] @ u[k] for k in range(3))
        out = np.zeros(self.plev[L].size)
        m = self.pmask(L)
        out[m] = r[m]
        return self.plev[L].sync(out)

    def divt(self, p, L, dst=None):
        """dst_k (inner velocity DoFs) = divT_k p; other DoFs of dst kept."""
        m = self.umask(L)
        out = [np.zeros(self.ulev[L].size) if dst is None else dst[k].copy() for k in range(3)]
        for k in range(3):
            out[k][m] = (self.B[L][k].T @ p)[m]
            self.ulev[L].sync(out[k])
        return out

    def velocity_apply(self, u, L, k):
        """Component k of the velocity block applied to u (all DoFs)."""
        if self.Vop is None:
            return self.Aop.A[L] @ u[k]
        return sum(self.Vop.A[L][k][j] @ u[j] for j in range(3))

    def apply(self, u, p, L):
        m = self.umask(L)
        du = []
        for k in range(3):
            r = self.velocity_apply(u, L, k) + self.B[L][k].T @ p
            o = np.zeros(self.ulev[L].size)
            o[m] = r[m]
            du.append(self.ulev[L].sync(o))
        return du, self.div(u, L)

    def residual(self, u, p, bu, bp, L):
        m = self.umask(L)
        ru = []
        for k in range(3):
            r = bu[k] - (self.velocity_apply(u, L, k) + self.B[L][k].T @ p)
            o = np.zeros(self.ulev[L].size)
            o[m] = r[m]
            ru.append(self.ulev[L].sync(o))
        rp = bp - self.div(u, L)
        mp = self.pmask(L)
        rp[~mp] = 0.0
        return ru, self.plev[L].sync(rp)

    def residual_norm(self, u, p, bu, bp, L):
        ru, rp = self.residual(u, p, bu, bp, L)
        m, mp = self.umask(L), self.pmask(L)
        return float(np.sqrt(sum((r[m] ** 2).sum() for r in ru) + (rp[mp] ** 2).sum()))

    # --- Uzawa smoother and multigrid ---------------------------------------------------------
    def uzawa(self, u, p, bu, bp, L, radius, order=3, sweeps=3, omega=0.7):
        m, mp = self.umask(L), self.pmask(L)
        ru = []
        for k in range(3):
            r = bu[k] - self.B[L][k].T @ p
            o = np.zeros(self.ulev[L].size)
            o[m] = r[m]
            ru.append(self.ulev[L].sync(o))
        u = [x.copy() for x in u]
        for _ in range(sweeps):
            if self.Vop is not None:
                u = _cheb_apply_vec(self.Vop, u, ru, L, radius, order)
                continue
            for k in range(3):
                u[k] = _cheb_apply(self.Aop, u[k], ru[k], L, radius, order)
        rp = bp - self.div(u, L)
        p = p.copy()
        p[mp] += omega * (self.sinv[L] * rp)[mp]
        return u, self.plev[L].sync(p)

    def vcycle(self, u, p, bu, bp, L, radii, order=3, pre=3, post=3, sweeps=3, omega=0.7, coarse=30):
        if L == self.minL:
            for _ in range(coarse):
                u, p = self.uzawa(u, p, bu, bp, L, radii[L], order, sweeps, omega)
            return u, p
        for _ in range(pre):
            u, p = self.uzawa(u, p, bu, bp, L, radii[L], order, sweeps, omega)
        ru, rp = self.residual(u, p, bu, bp, L)
        ucl, pcl = self.ulev[L - 1], self.plev[L - 1]
        bu_c = [self.utr.R[L] @ r for r in ru]
        bu_c = [self._mask_sync(ucl, v, self.umask(L - 1)) for v in bu_c]
        bp_c = self._mask_sync(pcl, self.ptr.R[L] @ rp, self.pmask(L - 1))
        uc = [np.zeros(ucl.size) for _ in range(3)]
        pc = np.zeros(pcl.size)
        uc, pc = self.vcycle(uc, pc, bu_c, bp_c, L - 1, radii, order, pre, post, sweeps, omega, coarse)
        m, mp = self.umask(L), self.pmask(L)
        u = [x.copy() for x in u]
        for k in range(3):
            u[k][m] += (self.utr.P[L] @ uc[k])[m]
            self.ulev[L].sync(u[k])
        p = p.copy()
        p[mp] += (self.ptr.P[L] @ pc)[mp]
        p = self.plev[L].sync(p)
        for _ in range(post):
            u, p = self.uzawa(u, p, bu, bp, L, radii[L], order, sweeps, omega)
        return u, p

    @staticmethod
    def _mask_sync(lev, v, m):
        o = np.zeros(lev.size)
        o[m] = v[m]
        return lev.sync(o)


def _cheb_apply_vec(op, x, b, L, radius, order):
    """_cheb_apply on the coupled velocity block (three components, block-diagonal D)."""
    x = [v.copy() for v in x]
    lev = op.levels[L]
    mask = lev.owned_mask(INNER | NEUMANN | FREESLIP)
    coeff = chebyshev_coefficients(order, 0.3 * radius, 1.2 * radius)
    tmp1, tmp2 = [v.copy() for v in x], [v.copy() for v in x]
    op.apply(x, tmp2, L, INNER | NEUMANN | FREESLIP)
    for k in range(3):
        tmp2[k][mask] = b[k][mask] - tmp2[k][mask]
        tmp1[k][mask] = op.invdiag[L][k][mask] * tmp2[k][mask]
        x[k][mask] = x[k][mask] + coeff[0] * tmp1[k][mask]
    for c in coeff[1:]:
        op.apply(tmp1, tmp2, L, INNER | NEUMANN | FREESLIP)
        for k in range(3):
            tmp1[k][mask] = op.invdiag[L][k][mask] * tmp2[k][mask]
            x[k][mask] = x[k][mask] + c * tmp1[k][mask]
    return x


def power_iteration_radius_vec(op, L, x0, iters):
    """power_iteration_radius on D^-1 A of the coupled velocity block (three components, flag All;
    norms and the Rayleigh quotient summed over the components)."""
    lev = op.levels[L]
    x = [v.copy() for v in x0]
    aux = [np.zeros_like(v) for v in x]
    m = lev.owned_mask(ALL)

    def dinv_a(src, dst):
        op.apply(src, dst, L, ALL)
        for k in range(3):
            dst[k][m] = op.invdiag[L][k][m] * dst[k][m]

    def vdot(a, b):
        return sum(dot(lev, a[k], b[k], ALL) for k in range(3))

    norm = math.sqrt(vdot(x, x))
    x = [v * (1.0 / norm) for v in x]
    dinv_a(x, aux)
    radius = 0.0
    for _ in range(iters):
        norm = math.sqrt(vdot(aux, aux))
        x = [v * (1.0 / norm) for v in aux]
        dinv_a(x, aux)
        radius = vdot(x, aux)
    return radius


def _cheb_apply(op, x, b, L, radius, order):
    """One ChebyshevSmoother application (as GMG.chebyshev_step, bounds 0.3 and 1.2 times the radius)."""
    x = x.copy()
    lev = op.levels[L]
    mask = lev.owned_mask(INNER | NEUMANN | FREESLIP)
    coeff = chebyshev_coefficients(order, 0.3 * radius, 1.2 * radius)
    tmp1, tmp2 = x.copy(), x.copy()
    op.apply(x, tmp2, L, INNER | NEUMANN | FREESLIP)
    tmp2[mask] = b[mask] - tmp2[mask]
    tmp1[mask] = op.invdiag[L][mask] * tmp2[mask]
    x[mask] = x[mask] + coeff[0] * tmp1[mask]
    for k in range(1, len(coeff)):
        op.apply(tmp1, tmp2, L, INNER | NEUMANN | FREESLIP)
        tmp1[mask] = op.invdiag[L][mask] * tmp2[mask]
        x[mask] = x[mask] + coeff[k] * tmp1[mask]
    return x
