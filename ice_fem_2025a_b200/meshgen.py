"""Synthetic tensor-product B-spline meshes in the reference's mesh format.

The reference reads its meshes from HDF5 files that a MATLAB generator writes
(TestCases/TriAxialCompression/Meshgen/GenerateMesh.m, SaveToHDF.m); those files are not
in the repository.  This module builds the same data for open, uniform, quadratic knot
vectors on a box:

* control points numbered x fastest (GenerateMesh.m:198-208),
* elements numbered x fastest, node-local order x fastest
  (``reshape(NodeNums(elConnU(u,:),elConnV(v,:),elConnW(w,:)),1,[])``, GenerateMesh.m:287-296),
* per-element Bezier extraction operators ``C = kron(Cz, kron(Cy, Cx))``
  (bezierExtraction3D.m:1-30), stored either as 1-D factors (``elem_kron``) or expanded
  (``elem_data``) exactly as ``elementgroup::AddElems`` holds ``ElemData(j,k)``
  (mesh/Groups/elementgroup.cpp:40-67).

The 1-D extraction operators follow the published algorithm of Borden, Scott, Evans and
Hughes, "Isogeometric finite element data structures based on Bezier extraction of NURBS",
IJNME 87 (2011), Algorithm 1.  Control points sit at the Greville abscissae, so the geometric
map is affine and elements are axis-aligned boxes.
"""
from __future__ import annotations

import dataclasses
import numpy as np


def open_uniform_knots(n_elem: int, p: int = 2) -> np.ndarray:
    inner = np.arange(1, n_elem) / n_elem
    return np.concatenate([np.zeros(p + 1), inner, np.ones(p + 1)])


def bezier_extraction_1d(knots: np.ndarray, p: int) -> np.ndarray:
    """Element extraction operators C[e] ((p+1)x(p+1)), N_local = C[e] @ B_bernstein."""
    U = np.asarray(knots, dtype=np.float64)
    m = len(U)
    a = p + 1
    b = a + 1
    ops = [np.eye(p + 1)]
    nb = 0
    while b < m:
        nxt = np.eye(p + 1)
        i = b
        while b < m and U[b] == U[b - 1]:
            b += 1
        mult = b - i + 1
        if mult < p:
            numer = U[b - 1] - U[a - 1]
            alphas = np.zeros(p + 1)
            for j in range(p, mult, -1):
                alphas[j - mult - 1] = numer / (U[a + j - 1] - U[a - 1])
            r = p - mult
            C = ops[nb]
            for j in range(1, r + 1):
                save = r - j + 1
                s = mult + j
                for k in range(p + 1, s, -1):
                    alpha = alphas[k - s - 1]
                    C[:, k - 1] = alpha * C[:, k - 1] + (1.0 - alpha) * C[:, k - 2]
                if b < m:
                    # C_next(save : j+save, save) = C(p-j+1 : p+1, p+1)   (1-based)
                    nxt[save - 1:j + save, save - 1] = C[p - j:p + 1, p]
        nb += 1
        ops.append(nxt)
        if b < m:
            a = b
            b += 1
    return np.stack(ops[:nb])


def greville(knots: np.ndarray, p: int) -> np.ndarray:
    n = len(knots) - p - 1
    return np.array([knots[i + 1:i + p + 1].mean() for i in range(n)])


@dataclasses.dataclass
class Mesh:
    dim: int
    elem_type: int            # 1 = B2_2, 2 = NURBS3_Cube2 (icefem_b200.h)
    coords: np.ndarray        # [n_nodes, dim]
    weights: np.ndarray | None
    elems: np.ndarray         # [n_elems, nen] int64
    elem_kron: np.ndarray     # [n_elems, dim, 3, 3]
    shape: tuple              # elements per direction
    elem_mat: np.ndarray | None = None
    full_data: np.ndarray | None = None   # explicit ElemData overriding the Kronecker factors

    @property
    def n_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.elems.shape[0])

    @property
    def nen(self) -> int:
        return int(self.elems.shape[1])

    def elem_data(self) -> np.ndarray:
        """Full extraction operators ElemData(j,k) = kron(Cz, kron(Cy, Cx)) [n_elems, nen, nen]."""
        if self.full_data is not None:
            return self.full_data
        k = self.elem_kron
        if self.dim == 2:
            # kron(Cy, Cx)[(ix+3iy),(jx+3jy)] = Cy[iy,jy] * Cx[ix,jx]
            C = np.einsum('eab,ecd->eacbd', k[:, 1], k[:, 0])   # (e, iy, ix, jy, jx)
            return C.reshape(self.n_elems, 9, 9)
        cyx = np.einsum('eab,ecd->eacbd', k[:, 1], k[:, 0]).reshape(self.n_elems, 9, 9)
        C = np.einsum('eab,ecd->eacbd', k[:, 2], cyx)            # (e, iz, iyx, jz, jyx)
        return C.reshape(self.n_elems, 27, 27)


def box_mesh(shape, lengths, p: int = 2, origin=None) -> Mesh:
    """Quadratic B-spline box mesh: shape = elements per direction, lengths = box size (m)."""
    if p != 2:
        raise ValueError("only quadratic meshes (B2_2 / NURBS3_Cube2) are supported")
    dim = len(shape)
    if dim not in (2, 3) or len(lengths) != dim:
        raise ValueError("shape/lengths must have 2 or 3 entries")
    origin = np.zeros(dim) if origin is None else np.asarray(origin, dtype=np.float64)
    ops, gr = [], []
    for n, L in zip(shape, lengths):
        kn = open_uniform_knots(n, p)
        ops.append(bezier_extraction_1d(kn, p))
        gr.append(greville(kn, p) * L)
    npts = [len(g) for g in gr]
    if dim == 2:
        nx, ny = npts
        gx, gy = np.meshgrid(gr[0], gr[1], indexing='xy')           # [ny, nx]
        coords = np.stack([gx.ravel(), gy.ravel()], axis=1) + origin
        ex, ey = np.meshgrid(np.arange(shape[0]), np.arange(shape[1]), indexing='xy')
        ex, ey = ex.ravel(), ey.ravel()
        lj, li = np.meshgrid(np.arange(3), np.arange(3), indexing='ij')   # li fastest
        li, lj = li.ravel(), lj.ravel()
        elems = (ex[:, None] + li[None, :]) + nx * (ey[:, None] + lj[None, :])
        kron = np.stack([ops[0][ex], ops[1][ey]], axis=1)
        weights = None
        etype = 1
    else:
        nx, ny, nz = npts
        gz, gy, gx = np.meshgrid(gr[2], gr[1], gr[0], indexing='ij')   # [nz, ny, nx]
        coords = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1) + origin
        ez, ey, ex = np.meshgrid(np.arange(shape[2]), np.arange(shape[1]), np.arange(shape[0]), indexing='ij')
        ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
        lk, lj, li = np.meshgrid(np.arange(3), np.arange(3), np.arange(3), indexing='ij')
        li, lj, lk = li.ravel(), lj.ravel(), lk.ravel()
        elems = ((ex[:, None] + li[None, :]) + nx * ((ey[:, None] + lj[None, :]) + ny * (ez[:, None] + lk[None, :])))
        kron = np.stack([ops[0][ex], ops[1][ey], ops[2][ez]], axis=1)
        weights = np.ones(coords.shape[0])
        etype = 2
    return Mesh(dim=dim, elem_type=etype, coords=np.ascontiguousarray(coords, dtype=np.float64),
                weights=weights, elems=np.ascontiguousarray(elems, dtype=np.int64),
                elem_kron=np.ascontiguousarray(kron, dtype=np.float64), shape=tuple(shape))


def _kron2(cs, cf):
    """kron(Cslow, Cfast) of 3x3 operators: index (i_fast + 3 i_slow, j_fast + 3 j_slow)."""
    return np.einsum('ab,cd->acbd', cs, cf).reshape(9, 9)


def box_face_groups(mesh: Mesh) -> dict:
    """Boundary element groups of a box mesh, built as the reference's generator builds them
    (TestCases/TriAxialCompression/Meshgen/GenerateMesh.m:298-367): "bottom" and "top" faces (x fastest, then y),
    "side" = front (y = min), back (y = max), left (x = min), right (x = max) faces, each with node-local order
    and extraction operator kron(C_slow, C_fast) of its two in-plane directions.  In 2D the groups are lines:
    "bottom"/"top" along x and "side" = left then right lines along y.  Returns {name: (faces, face_data)}."""
    ops = [bezier_extraction_1d(open_uniform_knots(n, 2), 2) for n in mesh.shape]
    npts = [n + 2 for n in mesh.shape]
    if mesh.dim == 2:
        ex, ey = mesh.shape
        nx, ny = npts
        num = lambda i, j: i + nx * j
        def line(fixed_axis, fixed, n_el, op):
            faces, data = [], []
            for e in range(n_el):
                idx = [e + a for a in range(3)]
                faces.append([num(fixed, k) if fixed_axis == 0 else num(k, fixed) for k in idx])
                data.append(op[e])
            return faces, data
        b = line(1, 0, ex, ops[0]); t = line(1, ny - 1, ex, ops[0])
        l = line(0, 0, ey, ops[1]); r = line(0, nx - 1, ey, ops[1])
        groups = {"bottom": b, "top": t, "side": (l[0] + r[0], l[1] + r[1])}
    else:
        ex, ey, ez = mesh.shape
        nx, ny, nz = npts
        num = lambda i, j, k: i + nx * (j + ny * k)
        def face(fix, val, slow_n, fast_n, slow_op, fast_op):
            faces, data = [], []
            for s_ in range(slow_n):
                for f_ in range(fast_n):
                    nodes = []
                    for b in range(3):          # slow direction
                        for a in range(3):      # fast direction
                            ijk = {"x": None, "y": None, "z": None}
                            ijk[fix] = val
                            free = [d for d in "xyz" if d != fix]
                            ijk[free[0]] = f_ + a
                            ijk[free[1]] = s_ + b
                            nodes.append(num(ijk["x"], ijk["y"], ijk["z"]))
                    faces.append(nodes)
                    data.append(_kron2(slow_op[s_], fast_op[f_]))
            return faces, data
        bot = face("z", 0, ey, ex, ops[1], ops[0]); top = face("z", nz - 1, ey, ex, ops[1], ops[0])
        fr = face("y", 0, ez, ex, ops[2], ops[0]); bk = face("y", ny - 1, ez, ex, ops[2], ops[0])
        le = face("x", 0, ez, ey, ops[2], ops[1]); ri = face("x", nx - 1, ez, ey, ops[2], ops[1])
        groups = {"bottom": bot, "top": top,
                  "side": (fr[0] + bk[0] + le[0] + ri[0], fr[1] + bk[1] + le[1] + ri[1])}
    return {k: (np.asarray(f, dtype=np.int64), np.asarray(d, dtype=np.float64)) for k, (f, d) in groups.items()}


def concat_meshes(meshes) -> Mesh:
    """Disjoint union (independent specimens); elem_mat = specimen index."""
    dim = meshes[0].dim
    coords, elems, kron, mats, w = [], [], [], [], []
    off = 0
    for i, m in enumerate(meshes):
        if m.dim != dim:
            raise ValueError("mixed dimensions")
        coords.append(m.coords)
        elems.append(m.elems + off)
        kron.append(m.elem_kron)
        mats.append(np.full(m.n_elems, i, dtype=np.int32))
        if m.weights is not None:
            w.append(m.weights)
        off += m.n_nodes
    return Mesh(dim=dim, elem_type=meshes[0].elem_type, coords=np.concatenate(coords),
                weights=np.concatenate(w) if w else None, elems=np.concatenate(elems),
                elem_kron=np.concatenate(kron), shape=(sum(m.n_elems for m in meshes),),
                elem_mat=np.concatenate(mats))
