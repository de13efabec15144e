"""CPU oracle for the cudolfinx assembly hot path (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import it.  The CUDA library must never route through it.

Parity status: **parity unpinned against DOLFINx** -- the reference publishes
no golden vectors and its own tests compare against DOLFINx at run time
(python/test/test_cuda_assembly.py:93-209); DOLFINx, FFCx, basix and PETSc
are not installed here, so the reference cannot be run.  The oracle is instead
pinned to closed-form known answers (tests/test_oracle.py): the P1 reference
stiffness matrix, exactly integrated reference tensors (rational arithmetic),
patch tests (linear fields are reproduced exactly), rigid-body modes of the
elasticity operator, and integral identities of the load vectors.

What it restates (reference file:line):

* mesh        -- unit cube, n^3 hexes x 6 tets sharing the v0-v7 diagonal, the
                 topology DOLFINx ``create_box(CellType.tetrahedron)`` produces
                 (python/examples/poisson.py:34-40).
* dofmaps     -- P1 = vertex numbering; P2 = vertices + edge midpoints with the
                 basix tetrahedron edge order (2,3),(1,3),(1,2),(0,3),(0,2),(0,1);
                 a blocked (bs=3) map is unrolled as ``dof*bs + comp``
                 (cpp/cudolfinx/fem/CUDADofMap.cpp:210-229).
* sparsity    -- sorted unique columns per row, block rows unrolled to scalar
                 AIJ (cpp/cudolfinx/la/petsc.cpp:38-65).
* matrix      -- per cell: element tensor, skip BC rows/cols, add into CSR
                 (cpp/cudolfinx/fem/CUDAFormIntegral.cpp:1154-1224), then set the
                 diagonal of BC rows (cpp/cudolfinx/fem/CUDAAssembler.cpp:131-164).
* vector      -- per cell element vector added into b
                 (cpp/cudolfinx/fem/CUDAFormIntegral.cpp:309-355).
* lifting     -- b[rows] -= scale * Ae[:, bc cols] (g - x0)[bc cols] for cells
                 with a BC column (cpp/cudolfinx/fem/CUDAFormIntegral.cpp:647-715).
* set_bc      -- b[d] = scale * (g[d] - x0[d]) for BC dofs
                 (cpp/cudolfinx/fem/CUDAAssembler.cpp:115-124).

Element tensors are computed from first principles (FFCx generates them in the
reference; they are exact for these polynomial integrands, so any exact
quadrature agrees up to rounding):

* P1 Poisson   Ae_ij = k_c |detJ|/6 grad(phi_i).grad(phi_j)   (k DG0 or 1)
* P2 Poisson   Ae_ij = sum_m k_m sum_ab G_ab R[m,a,b,i,j],  G = |detJ| K K^T,
               R = int_ref lambda_m d_a phi_i d_b phi_j     (k a P1 field)
* vector P2 elasticity (DG0 lambda, mu)
               A[(i,a),(j,b)] = mu (delta_ab S_ij + D[b,a,i,j]) + lam D[a,b,i,j]
               D[a,b,i,j] = int d_a phi_i d_b phi_j
* P1 load with P1 f:   b = M f,  M_ij = |detJ| (1 + delta_ij) / 120
* P2 load with DG0 f:  b_i = f_c |detJ| w_i, w = (-1/120 x4, 1/30 x6)
* vector P2 load with DG0 body force f_c (3 comps): b_(i,a) = f_ca |detJ| w_i
"""
from __future__ import annotations

from fractions import Fraction
from functools import lru_cache
from math import factorial

import numpy as np

# ---------------------------------------------------------------------------
# Reference-element tables (exact rational arithmetic, then cast to float64)
# ---------------------------------------------------------------------------

#: basix edge numbering of the reference tetrahedron
TET_EDGES = ((2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1))


def _mono_int(a, b, c):
    """int over the reference tet of x^a y^b z^c = a! b! c! / (a+b+c+3)!"""
    return Fraction(factorial(a) * factorial(b) * factorial(c), factorial(a + b + c + 3))


def _pmul(p, q):
    r = {}
    for k1, v1 in p.items():
        for k2, v2 in q.items():
            k = (k1[0] + k2[0], k1[1] + k2[1], k1[2] + k2[2])
            r[k] = r.get(k, 0) + v1 * v2
    return {k: v for k, v in r.items() if v != 0}


def _padd(p, q, s=1):
    r = dict(p)
    for k, v in q.items():
        r[k] = r.get(k, 0) + s * v
    return {k: v for k, v in r.items() if v != 0}


def _pscale(p, s):
    return {k: v * s for k, v in p.items()}


def _pdiff(p, ax):
    r = {}
    for k, v in p.items():
        if k[ax] > 0:
            kk = list(k)
            kk[ax] -= 1
            r[tuple(kk)] = r.get(tuple(kk), 0) + v * k[ax]
    return r


def _pint(p):
    return sum((v * _mono_int(*k) for k, v in p.items()), Fraction(0))


_LAMBDA = [
    {(0, 0, 0): Fraction(1), (1, 0, 0): Fraction(-1), (0, 1, 0): Fraction(-1), (0, 0, 1): Fraction(-1)},
    {(1, 0, 0): Fraction(1)},
    {(0, 1, 0): Fraction(1)},
    {(0, 0, 1): Fraction(1)},
]


def _basis(degree):
    if degree == 1:
        return list(_LAMBDA)
    if degree == 2:
        vert = [_pmul(l, _padd(_pscale(l, 2), {(0, 0, 0): Fraction(1)}, -1)) for l in _LAMBDA]
        edge = [_pscale(_pmul(_LAMBDA[a], _LAMBDA[b]), 4) for a, b in TET_EDGES]
        return vert + edge
    if degree == 3:
        # equispaced P3 Lagrange: vertices, two dofs per edge (basix edge
        # order, the point nearer the edge's first vertex first), face centroids
        one = {(0, 0, 0): Fraction(1)}
        two = {(0, 0, 0): Fraction(2)}
        vert = [_pscale(_pmul(l, _pmul(_padd(_pscale(l, 3), one, -1), _padd(_pscale(l, 3), two, -1))),
                        Fraction(1, 2)) for l in _LAMBDA]
        edge = []
        for a, b in TET_EDGES:
            ab = _pmul(_LAMBDA[a], _LAMBDA[b])
            edge.append(_pscale(_pmul(ab, _padd(_pscale(_LAMBDA[a], 3), one, -1)), Fraction(9, 2)))
            edge.append(_pscale(_pmul(ab, _padd(_pscale(_LAMBDA[b], 3), one, -1)), Fraction(9, 2)))
        face = [_pscale(_pmul(_pmul(_LAMBDA[a], _LAMBDA[b]), _LAMBDA[c]), 27)
                for a, b, c in ((1, 2, 3), (0, 2, 3), (0, 1, 3), (0, 1, 2))]
        return vert + edge + face
    raise ValueError(degree)


@lru_cache(maxsize=None)
def ref_grad_tensor(degree: int, weighted: bool):
    """R0[a,b,i,j] = int_ref d_a phi_i d_b phi_j   (weighted=False), shape (3,3,k,k)
    R[m,a,b,i,j] = int_ref lambda_m d_a phi_i d_b phi_j (weighted=True), (4,3,3,k,k)."""
    phi = _basis(degree)
    k = len(phi)
    dphi = [[_pdiff(p, ax) for ax in range(3)] for p in phi]
    if not weighted:
        out = np.zeros((3, 3, k, k))
        for a in range(3):
            for b in range(3):
                for i in range(k):
                    for j in range(k):
                        out[a, b, i, j] = float(_pint(_pmul(dphi[i][a], dphi[j][b])))
        return out
    out = np.zeros((4, 3, 3, k, k))
    for m in range(4):
        for a in range(3):
            for b in range(3):
                for i in range(k):
                    for j in range(k):
                        out[m, a, b, i, j] = float(_pint(_pmul(_LAMBDA[m], _pmul(dphi[i][a], dphi[j][b]))))
    return out


@lru_cache(maxsize=None)
def ref_mass_tensor(degree: int, weighted: bool):
    """M0[i,j] = int_ref phi_i phi_j (weighted=False), shape (k,k);
    M[m,i,j] = int_ref lambda_m phi_i phi_j (weighted=True), (4,k,k)."""
    phi = _basis(degree)
    k = len(phi)
    if not weighted:
        return np.array([[float(_pint(_pmul(phi[i], phi[j]))) for j in range(k)] for i in range(k)])
    return np.array([[[float(_pint(_pmul(_LAMBDA[m], _pmul(phi[i], phi[j])))) for j in range(k)]
                      for i in range(k)] for m in range(4)])


@lru_cache(maxsize=None)
def ref_basis_integrals(degree: int):
    """w_i = int_ref phi_i  (reference volume 1/6)."""
    return np.array([float(_pint(p)) for p in _basis(degree)])


# ---------------------------------------------------------------------------
# Exterior-facet reference tensors (ds integrals)
# ---------------------------------------------------------------------------
# facet i of a tetrahedron is the one opposite vertex i (basix / DOLFINx
# sub-entity numbering); the reference passes exterior facets as (cell, local
# facet) pairs (CUDAFormIntegral.cpp:361-447, active_mesh_entities).
TET_FACETS = ((1, 2, 3), (0, 2, 3), (0, 1, 3), (0, 1, 2))


def _bary_basis(degree):
    """Basis functions as polynomials in the four barycentric coordinates:
    dict {(e0, e1, e2, e3): coefficient}."""
    lam = [{tuple(1 if q == m else 0 for q in range(4)): Fraction(1)} for m in range(4)]

    def mul(p, q):
        r = {}
        for k1, v1 in p.items():
            for k2, v2 in q.items():
                k = tuple(a + b for a, b in zip(k1, k2))
                r[k] = r.get(k, 0) + v1 * v2
        return {k: v for k, v in r.items() if v != 0}

    if degree == 1:
        return lam, mul
    vert = []
    for m in range(4):
        p = {k: 2 * v for k, v in mul(lam[m], lam[m]).items()}
        for k, v in lam[m].items():
            p[k] = p.get(k, 0) - v
        vert.append(p)
    edge = [{k: 4 * v for k, v in mul(lam[a], lam[b]).items()} for a, b in TET_EDGES]
    return vert + edge, mul


def _facet_int(p, f):
    """int over facet f of p, divided by the facet area: barycentric monomials
    integrate to 2 a! b! c! / (a + b + c + 2)! on a triangle; lambda_f = 0 there."""
    tot = Fraction(0)
    for k, v in p.items():
        if k[f]:
            continue
        e = [k[m] for m in range(4) if m != f]
        tot += v * Fraction(2 * factorial(e[0]) * factorial(e[1]) * factorial(e[2]), factorial(sum(e) + 2))
    return tot


@lru_cache(maxsize=None)
def facet_ref_tensors(degree: int):
    """For each local facet f: mass M[f,i,j] = int_F phi_i phi_j / |F|,
    load l[f,i] = int_F phi_i / |F|, weighted load w[f,m,i] = int_F lambda_m phi_i / |F|."""
    phi, mul = _bary_basis(degree)
    lam = [{tuple(1 if q == m else 0 for q in range(4)): Fraction(1)} for m in range(4)]
    k = len(phi)
    M = np.zeros((4, k, k))
    l = np.zeros((4, k))
    w = np.zeros((4, 4, k))
    for f in range(4):
        for i in range(k):
            l[f, i] = float(_facet_int(phi[i], f))
            for j in range(k):
                M[f, i, j] = float(_facet_int(mul(phi[i], phi[j]), f))
            for m in range(4):
                w[f, m, i] = float(_facet_int(mul(lam[m], phi[i]), f))
    return M, l, w


def exterior_facets(cells):
    """(cell, local facet) pairs of the facets that belong to one cell only,
    ordered by cell then local facet."""
    F = np.sort(cells[:, np.array(TET_FACETS)], axis=2).reshape(-1, 3)
    _, inv, cnt = np.unique(F, axis=0, return_inverse=True, return_counts=True)
    ext = np.nonzero(cnt[inv.ravel()] == 1)[0]
    return np.stack([ext // 4, ext % 4], axis=1).astype(np.int32)


def facet_areas(coords, cells, facets):
    v = cells[facets[:, 0][:, None], np.array(TET_FACETS)[facets[:, 1]]]  # [F, 3]
    a, b, c = coords[v[:, 0]], coords[v[:, 1]], coords[v[:, 2]]
    return 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1)


def facet_mass(coords, cells, facets, degree, alpha=None):
    """Element matrices [F, k, k] of alpha * u * v * ds on cell-local dofs
    (alpha constant or one value per cell of the facet)."""
    M, _, _ = facet_ref_tensors(degree)
    area = facet_areas(coords, cells, facets)
    s = area if alpha is None else area * np.broadcast_to(np.asarray(alpha, dtype=float), area.shape)
    return s[:, None, None] * M[facets[:, 1]]


def facet_load(coords, cells, facets, degree, g=None, g_kind="constant", p1_cells=None):
    """Element vectors [F, k] of g * v * ds; g: constant, 'dg0' (one value per
    cell, indexed by the facet's cell) or 'p1' (vertex values; p1_cells gives
    the cells' P1 dofs)."""
    _, l, w = facet_ref_tensors(degree)
    area = facet_areas(coords, cells, facets)
    f = facets[:, 1]
    if g_kind == "p1":
        gv = np.asarray(g)[p1_cells[facets[:, 0]]]  # [F, 4]
        return area[:, None] * np.einsum("fm,fmi->fi", gv, w[f])
    if g_kind == "dg0":
        gc = np.asarray(g)[facets[:, 0]]
    else:
        gc = np.full(len(facets), 1.0 if g is None else float(g))
    return (area * gc)[:, None] * l[f]


def facet_vector_load(coords, cells, facets, t):
    """Element vectors [F, 30] (interleaved dof*3 + comp) of t . v ds on vector
    P2, t a constant 3-vector."""
    _, l, _ = facet_ref_tensors(2)
    area = facet_areas(coords, cells, facets)
    be = (area[:, None] * l[facets[:, 1]])[:, :, None] * np.asarray(t, dtype=float)[None, None, :]
    return be.reshape(len(facets), 30)


# ---------------------------------------------------------------------------
# Mesh and dofmaps
# ---------------------------------------------------------------------------

def unit_cube_tet_mesh(n: int, jitter: float = 0.0, seed: int = 0):
    """Unit cube split into n^3 hexes x 6 tetrahedra sharing the v0-v7 diagonal.

    Vertex (ix, iy, iz) has index iz*(n+1)^2 + iy*(n+1) + ix.  With ``jitter``
    > 0 every vertex moves by U[-jitter*h, jitter*h] per coordinate, except in
    the directions normal to the boundary planes it lies on (the domain stays
    the unit cube).  Returns (coords float64 [V,3], cells int32 [6 n^3, 4]).
    """
    n1 = n + 1
    g = np.arange(n1, dtype=np.float64) / n
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    coords = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-jitter / n, jitter / n, size=coords.shape)
        idx = np.stack(np.meshgrid(np.arange(n1), np.arange(n1), np.arange(n1), indexing="ij"), -1).reshape(-1, 3)[:, ::-1]
        on_bnd = (idx == 0) | (idx == n)
        d[on_bnd] = 0.0
        coords = coords + d
    iz, iy, ix = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    v0 = (iz * n1 * n1 + iy * n1 + ix).ravel()
    v1 = v0 + 1
    v2 = v0 + n1
    v3 = v1 + n1
    v4 = v0 + n1 * n1
    v5 = v1 + n1 * n1
    v6 = v2 + n1 * n1
    v7 = v3 + n1 * n1
    tets = [(v0, v1, v3, v7), (v0, v1, v7, v5), (v0, v5, v7, v4),
            (v0, v3, v2, v7), (v0, v6, v4, v7), (v0, v2, v6, v7)]
    cells = np.stack([np.stack(t, axis=1) for t in tets], axis=1).reshape(-1, 4)
    return coords, cells.astype(np.int32)


def vertex_grid_index(n: int):
    """(ix, iy, iz) integer grid index of every vertex (int64 [V,3])."""
    n1 = n + 1
    v = np.arange(n1 ** 3)
    return np.stack([v % n1, (v // n1) % n1, v // (n1 * n1)], axis=1)


def p2_dofmap(n: int, cells: np.ndarray):
    """P2 dofmap on the unit-cube mesh.

    Each dof sits on a point of the doubled grid (vertex 2*idx, edge midpoint
    idx_a + idx_b); dofs are numbered by lexicographic (z, y, x) order of those
    points, which interleaves vertex and edge dofs spatially.  Local order per
    cell: 4 vertices, then edges in basix order.  Returns (dofs int32 [C,10],
    num_dofs, doubled-grid index int64 [num_dofs,3]).
    """
    vg = vertex_grid_index(n)
    m = 2 * n + 1
    pts = [2 * vg[cells[:, v]] for v in range(4)]
    pts += [vg[cells[:, a]] + vg[cells[:, b]] for a, b in TET_EDGES]
    P = np.stack(pts, axis=1)  # [C,10,3]
    key = (P[..., 2] * m + P[..., 1]) * m + P[..., 0]
    uniq, inv = np.unique(key.ravel(), return_inverse=True)
    dofs = inv.reshape(key.shape).astype(np.int32)
    grid = np.stack([uniq % m, (uniq // m) % m, uniq // (m * m)], axis=1)
    return dofs, len(uniq), grid


def p3_local_points():
    """Barycentric weights (in thirds) of the 20 P3 nodes in local order."""
    w = [tuple(3 if q == v else 0 for q in range(4)) for v in range(4)]
    for a, b in TET_EDGES:
        w.append(tuple(2 if q == a else (1 if q == b else 0) for q in range(4)))
        w.append(tuple(1 if q == a else (2 if q == b else 0) for q in range(4)))
    for f in range(4):
        w.append(tuple(0 if q == f else 1 for q in range(4)))
    return np.array(w, dtype=np.int64)


def p3_dofmap(n: int, cells: np.ndarray):
    """Equispaced P3 dofmap on the unit-cube mesh: every node sits on the
    tripled grid (3x vertex index); dofs are numbered by lexicographic (z, y, x)
    order of the points that are nodes.  Returns (dofs int32 [C,20], num_dofs,
    tripled-grid index [num_dofs,3])."""
    vg = vertex_grid_index(n)
    m = 3 * n + 1
    W = p3_local_points()  # [20, 4]
    V = np.stack([vg[cells[:, v]] for v in range(4)], axis=1)  # [C,4,3]
    P = np.einsum("lv,cvd->cld", W, V)  # [C,20,3] tripled-grid coordinates
    key = (P[..., 2] * m + P[..., 1]) * m + P[..., 0]
    uniq, inv = np.unique(key.ravel(), return_inverse=True)
    dofs = inv.reshape(key.shape).astype(np.int32)
    grid = np.stack([uniq % m, (uniq // m) % m, uniq // (m * m)], axis=1)
    return dofs, len(uniq), grid


def boundary_dofs_from_grid(grid: np.ndarray, extent: int):
    """Dofs lying on the boundary of the unit cube: a grid coordinate equals 0
    or ``extent`` (exact topological marking for this structured mesh)."""
    return np.nonzero(np.any((grid == 0) | (grid == extent), axis=1))[0].astype(np.int32)


def dof_coordinates(coords, cells, dofs, num_dofs, degree):
    """Physical coordinates of each dof (vertex or edge midpoint)."""
    X = np.zeros((num_dofs, 3))
    if degree == 1:
        X[dofs.ravel()] = coords[cells.ravel()]
        return X
    cc = coords[cells]  # [C,4,3]
    if degree == 3:
        P = np.einsum("lv,cvd->cld", p3_local_points() / 3.0, cc)
        X[dofs.ravel()] = P.reshape(-1, 3)
        return X
    pts = [cc[:, v] for v in range(4)] + [0.5 * (cc[:, a] + cc[:, b]) for a, b in TET_EDGES]
    P = np.stack(pts, axis=1)
    X[dofs.ravel()] = P.reshape(-1, 3)
    return X


# ---------------------------------------------------------------------------
# Sparsity (cpp/cudolfinx/la/petsc.cpp:38-65; DOLFINx SparsityPattern)
# ---------------------------------------------------------------------------

def block_sparsity(dofs0, dofs1, n0):
    """Sorted unique block columns per block row: returns (bptr, bcol)."""
    k0, k1 = dofs0.shape[1], dofs1.shape[1]
    r = np.repeat(dofs0, k1, axis=1).astype(np.int64).ravel()
    c = np.tile(dofs1, (1, k0)).astype(np.int64).ravel()
    ncol = int(dofs1.max()) + 1 if dofs1.size else 1
    key = np.unique(r * ncol + c)
    rows = key // ncol
    cols = (key % ncol).astype(np.int32)
    bptr = np.zeros(n0 + 1, dtype=np.int64)
    np.add.at(bptr, rows + 1, 1)
    return np.cumsum(bptr), cols


def sparsity(dofs0, dofs1, n0, bs0=1, bs1=1):
    """Scalar (unrolled) CSR pattern: row bs0*R+a has columns bs1*C+b for C in
    the sorted block columns of R and b in 0..bs1-1 (la/petsc.cpp:45-65)."""
    bptr, bcol = block_sparsity(dofs0, dofs1, n0)
    blen = np.diff(bptr)
    row_len = np.repeat(blen * bs1, bs0)
    row_ptr = np.zeros(n0 * bs0 + 1, dtype=np.int64)
    row_ptr[1:] = np.cumsum(row_len)
    # unrolled columns of each block row, repeated bs0 times
    ucol = (bcol.astype(np.int64)[:, None] * bs1 + np.arange(bs1)[None, :]).ravel()
    col = np.empty(row_ptr[-1], dtype=np.int32)
    # each scalar row bs0*R+a copies ucol[bptr[R]*bs1 : bptr[R+1]*bs1]
    seg_start = np.repeat(bptr[:-1] * bs1, bs0)  # start of source segment for each scalar row
    seg_len = row_len
    total = int(row_ptr[-1])
    if total:
        rid = np.repeat(np.arange(n0 * bs0), seg_len)
        off = np.arange(total) - row_ptr[rid]
        col[:] = ucol[seg_start[rid] + off]
    return row_ptr.astype(np.int32), col


def diag_positions(row_ptr, col):
    """Slot of A[r, r] in CSR for every row (-1 if absent)."""
    nrows = len(row_ptr) - 1
    out = np.full(nrows, -1, dtype=np.int64)
    rid = np.repeat(np.arange(nrows), np.diff(row_ptr))
    hit = np.nonzero(col == rid)[0]
    out[rid[hit]] = hit
    return out


def csr_slots(row_ptr, col, rows, cols):
    """Slot index of (rows[i], cols[i]) via binary search in each CSR row
    (the reference's ``binary_search``, CUDAFormIntegral.cpp:2572-2602)."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    rp = row_ptr.astype(np.int64)
    # global key search: rows are sorted blocks, columns sorted inside a row
    key_all = np.repeat(np.arange(len(rp) - 1, dtype=np.int64), np.diff(rp)) * (1 << 32) + col.astype(np.int64)
    key = rows * (1 << 32) + cols
    s = np.searchsorted(key_all, key)
    ok = (s < len(key_all)) & (key_all[np.minimum(s, len(key_all) - 1)] == key)
    if not np.all(ok):
        raise KeyError("entry not in sparsity pattern")
    return s


# ---------------------------------------------------------------------------
# Geometry
# ---------------------------------------------------------------------------

def cell_geometry(coords, cells):
    """Per cell: J (C,3,3) with columns x_k - x_0, detJ (C,), K = J^{-1} (C,3,3)."""
    x = coords[cells]  # [C,4,3]
    J = np.stack([x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]], axis=2)
    det = np.linalg.det(J)
    K = np.linalg.inv(J)
    return J, det, K


# ---------------------------------------------------------------------------
# Element tensors (first principles; FFCx tabulate_tensor in the reference)
# ---------------------------------------------------------------------------

_P1_REF_GRAD = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


def p1_stiffness(coords, cells, k_dg0=None):
    """Ae [C,4,4] of k * inner(grad u, grad v) * dx with P1, k DG0 (or 1)."""
    _, det, K = cell_geometry(coords, cells)
    G = np.einsum("ia,cab->cib", _P1_REF_GRAD, K)  # grad phi_i = K^T ghat_i  -> (ghat K)_b
    Ae = np.abs(det)[:, None, None] / 6.0 * np.einsum("cib,cjb->cij", G, G)
    if k_dg0 is not None:
        Ae = Ae * np.asarray(k_dg0)[:, None, None]
    return Ae


def p2_stiffness(coords, cells, k_cell_values):
    """Ae [C,10,10] of k * inner(grad u, grad v) * dx with P2, k a P1 field
    given by its 4 vertex values per cell ``k_cell_values`` [C,4]."""
    _, det, K = cell_geometry(coords, cells)
    G = np.abs(det)[:, None, None] * np.einsum("cak,cbk->cab", K, K)
    R = ref_grad_tensor(2, True)  # [4,3,3,10,10]
    return np.einsum("cm,cab,mabij->cij", k_cell_values, G, R, optimize=True)


def p3_stiffness(coords, cells, k_dg0=None):
    """Ae [C,20,20] of k * inner(grad u, grad v) * dx with equispaced P3, k DG0 (or 1)."""
    _, det, K = cell_geometry(coords, cells)
    G = np.abs(det)[:, None, None] * np.einsum("cak,cbk->cab", K, K)
    R0 = ref_grad_tensor(3, False)  # [3,3,20,20]
    Ae = np.einsum("cab,abij->cij", G, R0, optimize=True)
    if k_dg0 is not None:
        Ae = Ae * np.asarray(k_dg0)[:, None, None]
    return Ae


def mass_matrices(coords, cells, degree, c_dg0=None, c_vertex=None):
    """Ae [C,k,k] of c * u * v * dx on P1/P2: c = 1, DG0 per cell (``c_dg0``) or
    a P1 field given by its 4 vertex values per cell (``c_vertex`` [C,4]).
    The reference assembles such forms from FFCx kernels
    (CUDAFormIntegral.cpp:1103-1226); here the reference mass tensors are
    integrated exactly."""
    _, det, _ = cell_geometry(coords, cells)
    adet = np.abs(det)
    if c_vertex is not None:
        return np.einsum("c,cm,mij->cij", adet, np.asarray(c_vertex), ref_mass_tensor(degree, True), optimize=True)
    c = adet if c_dg0 is None else adet * np.asarray(c_dg0)
    return c[:, None, None] * ref_mass_tensor(degree, False)[None]


def vector_mass(Ae_scalar, bs=3):
    """Ae [C, k*bs, k*bs] of rho * inner(u, v) * dx from the scalar mass
    matrices: local index i*bs + a couples with j*bs + a only."""
    C, k, _ = Ae_scalar.shape
    out = np.zeros((C, k, bs, k, bs))
    for a in range(bs):
        out[:, :, a, :, a] = Ae_scalar
    return out.reshape(C, k * bs, k * bs)


def p3_load_dg0(coords, cells, f_cell):
    """be [C,20] of f * v * dx with f DG0: |det| f int_ref phi_i."""
    _, det, _ = cell_geometry(coords, cells)
    return (np.abs(det) * np.asarray(f_cell))[:, None] * ref_basis_integrals(3)[None, :]


def p2_elasticity(coords, cells, lam, mu):
    """Ae [C,30,30] (local index 3*i + a) of 2 mu eps(u):eps(v) + lam div u div v,
    vector P2, DG0 lam and mu."""
    _, det, K = cell_geometry(coords, cells)
    R0 = ref_grad_tensor(2, False)  # [3,3,10,10]
    # D[a,b,i,j] = |det| sum_{al,be} K[al,a] K[be,b] R0[al,be,i,j]
    D = np.abs(det)[:, None, None, None, None] * np.einsum("cpa,cqb,pqij->cabij", K, K, R0, optimize=True)
    S = np.einsum("caaij->cij", D)
    C = len(cells)
    A = np.zeros((C, 10, 3, 10, 3))
    eye = np.eye(3)
    # mu (delta_ab S_ij + D[b,a,i,j]) + lam D[a,b,i,j]
    A += mu[:, None, None, None, None] * (eye[None, None, :, None, :] * S[:, :, None, :, None])
    A += mu[:, None, None, None, None] * np.transpose(D, (0, 3, 2, 4, 1))   # D[b,a,i,j] at [i,a,j,b]
    A += lam[:, None, None, None, None] * np.transpose(D, (0, 3, 1, 4, 2))  # D[a,b,i,j] at [i,a,j,b]
    return A.reshape(C, 30, 30)


def p1_load_p1f(coords, cells, f_vertex):
    """be [C,4] of f*v*dx with f a P1 field (vertex values), P1 test space."""
    _, det, _ = cell_geometry(coords, cells)
    fc = f_vertex[cells]
    return np.abs(det)[:, None] / 120.0 * (fc + fc.sum(axis=1, keepdims=True))


def p2_load_dg0(coords, cells, f_cell):
    """be [C,10] of f*v*dx with f DG0, P2 test space."""
    _, det, _ = cell_geometry(coords, cells)
    w = ref_basis_integrals(2)
    return (np.abs(det) * f_cell)[:, None] * w[None, :]


def p2_vector_load_dg0(coords, cells, f_cell3):
    """be [C,30] (index 3*i + a) of inner(f, v)*dx, f DG0 vector [C,3]."""
    _, det, _ = cell_geometry(coords, cells)
    w = ref_basis_integrals(2)
    be = np.abs(det)[:, None, None] * w[None, :, None] * f_cell3[:, None, :]
    return be.reshape(len(cells), 30)


# ---------------------------------------------------------------------------
# Global assembly
# ---------------------------------------------------------------------------

def unroll(dofs, bs):
    """dof*bs + comp (CUDADofMap.cpp:227)."""
    if bs == 1:
        return dofs.astype(np.int64)
    return (dofs.astype(np.int64)[:, :, None] * bs + np.arange(bs)).reshape(len(dofs), -1)


def assemble_matrix(Ae, dofs0, dofs1, row_ptr, col, bs0=1, bs1=1,
                    bc0_markers=None, bc1_markers=None, diagonal=1.0, bc0_owned_dofs=None):
    """CSR values: sum_e Ae scattered with BC rows/cols skipped
    (CUDAFormIntegral.cpp:1195-1213), then A[d,d] = diagonal for BC rows
    (CUDAAssembler.cpp:131-164)."""
    u0 = unroll(dofs0, bs0)
    u1 = unroll(dofs1, bs1)
    C, k0 = u0.shape
    k1 = u1.shape[1]
    rows = np.repeat(u0, k1, axis=1).ravel()
    cols = np.tile(u1, (1, k0)).ravel()
    vals = Ae.reshape(C, k0 * k1).ravel()
    keep = np.ones(rows.shape, dtype=bool)
    if bc0_markers is not None:
        keep &= bc0_markers[rows] == 0
    if bc1_markers is not None:
        keep &= bc1_markers[cols] == 0
    slots = csr_slots(row_ptr, col, rows[keep], cols[keep])
    values = np.zeros(len(col))
    np.add.at(values, slots, vals[keep])
    if bc0_owned_dofs is not None and len(bc0_owned_dofs):
        dpos = diag_positions(row_ptr, col)
        d = dpos[np.asarray(bc0_owned_dofs)]
        values[d[d >= 0]] = diagonal
    return values


def assemble_vector(be, dofs, num_values, bs=1):
    """b += be scattered (CUDAFormIntegral.cpp:345-354)."""
    u = unroll(dofs, bs)
    b = np.zeros(num_values)
    np.add.at(b, u.ravel(), be.reshape(-1))
    return b


def assemble_diagonal(Ae, dofs, num_values, bs=1):
    """Vector of the bilinear form's diagonal, b[r] += Ae[r][r] over the cells,
    no BCs: what a form compiled with FFCx's ``"part": "diagonal"`` assembles
    (python/test/test_cuda_assembly.py:199-208).  It equals the diagonal of
    the matrix assembled without BCs."""
    return assemble_vector(np.diagonal(Ae, axis1=1, axis2=2), dofs, num_values, bs)


def apply_lifting(b, Ae, dofs0, dofs1, bc1_markers, g, x0=None, scale=1.0, bs0=1, bs1=1):
    """b -= scale * A (g - x0) restricted to BC columns, for every cell with a
    BC column (CUDAFormIntegral.cpp:647-715)."""
    u0 = unroll(dofs0, bs0)
    u1 = unroll(dofs1, bs1)
    m = bc1_markers[u1] != 0
    has = np.nonzero(m.any(axis=1))[0]
    if len(has) == 0:
        return b
    u0h, u1h, mh = u0[has], u1[has], m[has]
    d = g[u1h] - (x0[u1h] if x0 is not None else 0.0)
    d = np.where(mh, d, 0.0)
    be = -scale * np.einsum("cij,cj->ci", Ae[has], d)
    np.add.at(b, u0h.ravel(), be.ravel())
    return b


def set_bc(b, bc_dofs, g, x0=None, scale=1.0):
    """b[d] = scale * (g[d] - x0[d]) (CUDAAssembler.cpp:115-124)."""
    d = np.asarray(bc_dofs)
    b[d] = scale * (g[d] - (x0[d] if x0 is not None else 0.0))
    return b


# ---------------------------------------------------------------------------
# Parity bounds: how far an assembled entry may lie from the oracle's
# ---------------------------------------------------------------------------
#
# An assembled entry is a sum of element contributions added in an order the
# reference leaves open (FP64 atomics, CUDAFormIntegral.cpp:1154-1224).  Its
# bound is per entry: PARITY_RTOL times the sum of the |contributions| (the
# reordering error of a sum is at most (m-1) u sum|c_i|, u = 2^-53, far below
# 1e-12 for the m <= 100 contributions of these meshes), plus PARITY_FREL
# times the largest |entry| of each contributing element (the element
# tensor's own rounding: an entry that is zero or cancels inside one element
# is computed to a few ulps of that element's scale, which depends on the
# element's coefficient and size, never on the rest of the matrix).  Entries
# nothing contributes to, and the values written by set_diagonal / set_bc,
# have bound 0: they must match exactly.

PARITY_RTOL = 1e-12
PARITY_FREL = 1e-14


def _element_floor(T):
    """Largest |entry| of each element tensor T [C, ...]."""
    T = np.abs(np.asarray(T))
    return T.reshape(len(T), -1).max(axis=1) if len(T) else np.zeros(0)


def matrix_bound(Ae, dofs0, dofs1, row_ptr, col, bs0=1, bs1=1, bc0_markers=None, bc1_markers=None,
                 rtol=PARITY_RTOL, frel=PARITY_FREL):
    """Per-slot parity bound of assemble_matrix(Ae, ...): the same scatter of
    rtol*|Ae| + frel*max|Ae_cell| (BC rows / columns skipped, so BC rows --
    whose diagonal set_diagonal writes -- have bound 0)."""
    Ae = np.asarray(Ae)
    contrib = rtol * np.abs(Ae) + frel * _element_floor(Ae).reshape((-1,) + (1,) * (Ae.ndim - 1))
    return assemble_matrix(contrib, dofs0, dofs1, row_ptr, col, bs0, bs1, bc0_markers, bc1_markers)


def vector_bound(be, dofs, num_values, bs=1, rtol=PARITY_RTOL, frel=PARITY_FREL):
    """Per-entry parity bound of assemble_vector(be, ...)."""
    be = np.asarray(be)
    contrib = rtol * np.abs(be) + frel * _element_floor(be).reshape((-1,) + (1,) * (be.ndim - 1))
    return assemble_vector(contrib, dofs, num_values, bs)


def lifting_bound(num_values, Ae, dofs0, dofs1, bc1_markers, g, x0=None, scale=1.0, bs0=1, bs1=1,
                  rtol=PARITY_RTOL, frel=PARITY_FREL):
    """Per-entry parity bound of apply_lifting: for row i of a cell with BC
    columns, rtol*|scale|*sum_j |Ae_ij d_j| + frel*|scale|*max|Ae_cell|*sum_j |d_j|
    (d = g - x0 on the cell's BC columns)."""
    u0 = scalar_cell_dofs(dofs0, bs0)  # -1 outside a restriction
    u1 = scalar_cell_dofs(dofs1, bs1)
    out = np.zeros(num_values)
    m = (u1 >= 0) & (np.asarray(bc1_markers)[np.maximum(u1, 0)] != 0)
    has = np.nonzero(m.any(axis=1))[0]
    if len(has) == 0:
        return out
    u0h, u1h, mh = u0[has], np.maximum(u1[has], 0), m[has]
    d = np.abs(np.where(mh, g[u1h] - (x0[u1h] if x0 is not None else 0.0), 0.0))
    A = np.abs(np.asarray(Ae)[has])
    per_row = rtol * np.einsum("cij,cj->ci", A, d) + (frel * _element_floor(A) * d.sum(axis=1))[:, None]
    keep = u0h >= 0
    np.add.at(out, u0h[keep], abs(scale) * per_row[keep])
    return out


def diagonal_bound(Ae, dofs, num_values, bs=1, rtol=PARITY_RTOL, frel=PARITY_FREL):
    """Per-entry parity bound of assemble_diagonal: rtol*|Ae_ii| + frel*max|Ae_cell|."""
    Ae = np.asarray(Ae)
    contrib = rtol * np.abs(np.diagonal(Ae, axis1=1, axis2=2)) + frel * _element_floor(Ae)[:, None]
    return assemble_vector(contrib, dofs, num_values, bs)


def within_bound(gpu, ref, bound):
    """(all |gpu - ref| <= bound, worst |gpu - ref| / bound); a nonzero
    difference where the bound is 0 counts as infinitely far."""
    gpu = np.asarray(gpu, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    bound = np.broadcast_to(np.asarray(bound, dtype=np.float64), ref.shape)
    err = np.abs(gpu - ref)
    ok = bool(np.all(err <= bound))
    if not err.size:
        return ok, 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.where(err == 0.0, 0.0, err / bound)
    return ok, float(np.max(ratio))


# ---------------------------------------------------------------------------
# Block / restricted systems (python/cudolfinx/form.py:107-225,
# assemble.py:112-202, cpp/cudolfinx/fem/petsc.h:39-107, fem/utils.h:14-98)
# ---------------------------------------------------------------------------

def restricted_dofmap(dofs, restriction, num_blocks):
    """Cell dofs renumbered to their position in `restriction` (sorted kept
    block dofs), -1 outside it (CUDADofMap::update with a restriction map,
    cpp/cudolfinx/fem/CUDADofMap.cpp:199-236)."""
    remap = np.full(num_blocks, -1, dtype=np.int64)
    remap[np.asarray(restriction)] = np.arange(len(restriction))
    return remap[np.asarray(dofs)]


def scalar_cell_dofs(dofs, bs):
    """[C, k*bs] scalar dofs dof*bs + comp, -1 where the block dof is -1."""
    d = np.asarray(dofs, dtype=np.int64)
    s = (d[:, :, None] * bs + np.arange(bs)).reshape(d.shape[0], -1)
    s[np.repeat(d < 0, bs, axis=1)] = -1
    return s


def _couplings(d0, d1, bs0, bs1):
    s0, s1 = scalar_cell_dofs(d0, bs0), scalar_cell_dofs(d1, bs1)
    R = np.broadcast_to(s0[:, :, None], (s0.shape[0], s0.shape[1], s1.shape[1]))
    C = np.broadcast_to(s1[:, None, :], R.shape)
    return R, C, (R >= 0) & (C >= 0)


def block_pattern(parts, num_rows, num_cols):
    """Monolithic scalar CSR of a block system: the union of every part's cell
    couplings placed at its offsets, sorted unique columns per row (DOLFINx's
    block SparsityPattern at block size 1, as create_cuda_matrix_block builds
    it, cpp/cudolfinx/fem/petsc.h:39-107; restricted couplings as in
    compute_restricted_sparsity_pattern, fem/utils.h:14-98).
    parts = [(dofs0, dofs1, bs0, bs1, row_offset, col_offset)], -1 = excluded."""
    keys = [np.zeros(0, dtype=np.int64)]
    for d0, d1, bs0, bs1, ro, co in parts:
        R, C, m = _couplings(d0, d1, bs0, bs1)
        keys.append((ro + R[m]) * num_cols + (co + C[m]))
    k = np.unique(np.concatenate(keys))
    rows, cols = k // num_cols, k % num_cols
    row_ptr = np.zeros(num_rows + 1, dtype=np.int64)
    np.add.at(row_ptr, rows + 1, 1)
    return np.cumsum(row_ptr).astype(np.int32), cols.astype(np.int32)


def assemble_block_matrix(blocks, row_ptr, col, diagonal=1.0):
    """Monolithic values of a block system: each block (a dict with Ae
    [C, k0*bs0, k1*bs1], dofs0, dofs1, bs0, bs1, row_offset, col_offset and
    optional markers0 / markers1 / bc_rows in its own, restricted numbering)
    adds its element matrices at its offsets, skipping excluded dofs and
    BC-marked rows / columns (the per-block assemble_matrix calls of
    assemble_matrix_block, assemble.py:112-134, each a
    CUDAFormIntegral.cpp:1154-1224 scatter); then every block's BC rows get
    `diagonal` on the monolithic diagonal (CUDAAssembler.cpp:131-164)."""
    values = np.zeros(len(col))
    dpos = diag_positions(row_ptr, col)
    for B in blocks:
        R, C, m = _couplings(B["dofs0"], B["dofs1"], B["bs0"], B["bs1"])
        m = m.copy()
        if B.get("markers0") is not None:
            m &= np.asarray(B["markers0"])[np.maximum(R, 0)] == 0
        if B.get("markers1") is not None:
            m &= np.asarray(B["markers1"])[np.maximum(C, 0)] == 0
        slots = csr_slots(row_ptr, col, B["row_offset"] + R[m], B["col_offset"] + C[m])
        np.add.at(values, slots, np.asarray(B["Ae"])[m])
    for B in blocks:
        if B.get("bc_rows") is not None and len(B["bc_rows"]):
            d = dpos[B["row_offset"] + np.asarray(B["bc_rows"], dtype=np.int64)]
            values[d[d >= 0]] = diagonal
    return values


def block_matrix_bound(blocks, row_ptr, col, rtol=PARITY_RTOL, frel=PARITY_FREL):
    """Per-slot parity bound of assemble_block_matrix (the bound of
    matrix_bound for every block at its offsets; 0 on the BC diagonals)."""
    bb = []
    for B in blocks:
        Ae = np.asarray(B["Ae"])
        c = dict(B)
        c["Ae"] = rtol * np.abs(Ae) + frel * _element_floor(Ae).reshape((-1,) + (1,) * (Ae.ndim - 1))
        bb.append(c)
    return assemble_block_matrix(bb, row_ptr, col, diagonal=0.0)


def block_vector_bound(parts, size, rtol=PARITY_RTOL, frel=PARITY_FREL):
    """Per-entry parity bound of assemble_block_vector."""
    out = []
    for be, dofs, bs, off in parts:
        be = np.asarray(be)
        out.append((rtol * np.abs(be) + frel * _element_floor(be).reshape((-1,) + (1,) * (be.ndim - 1)), dofs,
                    bs, off))
    return assemble_block_vector(out, size)


def assemble_block_vector(parts, size):
    """Monolithic vector: part (be [C, k*bs], dofs, bs, offset) adds its element
    vectors at its offset, skipping excluded dofs (assemble_vector_block,
    assemble.py:168-202)."""
    b = np.zeros(size)
    for be, dofs, bs, off in parts:
        s = scalar_cell_dofs(dofs, bs)
        m = s >= 0
        np.add.at(b, off + s[m], np.asarray(be).reshape(s.shape)[m])
    return b


# ---------------------------------------------------------------------------
# Interior-facet (dS) integrals of discontinuous spaces
# (CUDAFormIntegral.cpp:451-522 vector, :1988-2103 matrix)
# ---------------------------------------------------------------------------

def interior_facets(cells):
    """(cell0, local facet0, cell1, local facet1) of every facet shared by two
    cells, cell0 < cell1, ordered by the facet's sorted vertex triple."""
    F = np.sort(cells[:, np.array(TET_FACETS)], axis=2).reshape(-1, 3)
    _, inv, cnt = np.unique(F, axis=0, return_inverse=True, return_counts=True)
    inv = inv.ravel()
    order = np.argsort(inv, kind="stable")
    start = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    two = np.nonzero(cnt == 2)[0]
    e0, e1 = order[start[two]], order[start[two] + 1]
    return np.stack([e0 // 4, e0 % 4, e1 // 4, e1 % 4], axis=1).astype(np.int32)


def dg_dofmap(num_cells, degree):
    """Discontinuous Lagrange dofmap: each cell owns its dofs (DG0: one, DG1:
    one per vertex in the cell's vertex order)."""
    k = 1 if degree == 0 else 4
    return np.arange(num_cells * k, dtype=np.int32).reshape(num_cells, k)


def _barycentric(coords, cells, c, X):
    """Barycentric coordinates [F, q, 4] of points X [F, q, 3] in cells c [F]."""
    x = coords[cells[c]]  # [F,4,3]
    J = np.transpose(x[:, 1:] - x[:, :1], (0, 2, 1))  # columns x_k - x_0
    l = np.linalg.solve(J[:, None], (X - x[:, :1])[..., None])[..., 0]
    return np.concatenate([1.0 - l.sum(axis=2, keepdims=True), l], axis=2)


def _facet_traces(coords, cells, quads, degree):
    """Quadrature (the 3 edge midpoints of the facet, weight area/3 each:
    exact for quadratics) and the traces of both cells' bases there:
    returns w [F, 3], T0 [F, 3, k], T1 [F, 3, k]."""
    quads = np.asarray(quads)
    c0, f0, c1 = quads[:, 0], quads[:, 1], quads[:, 2]
    v = cells[c0[:, None], np.array(TET_FACETS)[f0]]  # [F,3] facet vertices
    P = coords[v]  # [F,3,3]
    X = 0.5 * (P + P[:, [1, 2, 0]])  # edge midpoints
    area = 0.5 * np.linalg.norm(np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), axis=1)
    w = np.repeat(area[:, None] / 3.0, 3, axis=1)
    if degree == 0:
        one = np.ones((len(quads), 3, 1))
        return w, one, one
    return w, _barycentric(coords, cells, c0, X), _barycentric(coords, cells, c1, X)


def interior_jump_tensors(coords, cells, quads, degree, alpha=None):
    """[F, 2k, 2k] of alpha * jump(u) * jump(v) * dS: macro dofs = cell0's
    then cell1's, jump = trace from cell0 minus trace from cell1; alpha per
    facet (the DG0 average of the two cells, or 1)."""
    w, T0, T1 = _facet_traces(coords, cells, quads, degree)
    S = np.concatenate([T0, -T1], axis=2)  # [F,3,2k]
    A = np.einsum("fq,fqi,fqj->fij", w, S, S)
    return A if alpha is None else A * np.asarray(alpha)[:, None, None]


def interior_avg_load(coords, cells, quads, degree, g=None):
    """[F, 2k] of g * avg(v) * dS (g per facet, or 1)."""
    w, T0, T1 = _facet_traces(coords, cells, quads, degree)
    be = 0.5 * np.einsum("fq,fqi->fi", w, np.concatenate([T0, T1], axis=2))
    return be if g is None else be * np.asarray(g)[:, None]


def interior_jump_norm(coords, cells, quads, degree, u_macro):
    """sum over the facets of int jump(u)^2 dS, u_macro [F, 2k] the macro dof values."""
    w, T0, T1 = _facet_traces(coords, cells, quads, degree)
    S = np.concatenate([T0, -T1], axis=2)
    return float(np.einsum("fq,fq->", w, np.einsum("fqi,fi->fq", S, u_macro) ** 2))


def macro_dofmap(dofs, quads):
    """[F, 2k]: cell0's dofs then cell1's for every interior facet."""
    quads = np.asarray(quads)
    return np.concatenate([dofs[quads[:, 0]], dofs[quads[:, 2]]], axis=1)


def facet_average(values_per_cell, quads):
    """The average of a DG0 field over the two cells of each interior facet."""
    v = np.asarray(values_per_cell)
    return 0.5 * (v[quads[:, 0]] + v[quads[:, 2]])


# ---------------------------------------------------------------------------
# Same-map interpolation (cpp/cudolfinx/fem/CUDACoefficient.h:64-83,
# cpp/cudolfinx/fem/CUDAInterpolate.cu)
# ---------------------------------------------------------------------------

def element_nodes(degree):
    """Reference coordinates [k, 3] of the Lagrange nodes in local order;
    degree 0 = DG0 (the centroid)."""
    if degree == 0:
        return np.full((1, 3), 0.25)
    if degree == 1:
        B = np.eye(4)
    elif degree == 2:
        B = np.array([np.eye(4)[v] for v in range(4)] + [0.5 * (np.eye(4)[a] + np.eye(4)[b]) for a, b in TET_EDGES])
    else:
        B = p3_local_points() / 3.0
    return B[:, 1:]


def interpolation_operator(degree_target, degree_source):
    """[k1, k0]: the target nodes evaluated in the source basis (the exact
    rational basis of this module; create_interpolation_operator for Lagrange
    elements)."""
    X = element_nodes(degree_target)
    if degree_source == 0:
        return np.ones((len(X), 1))
    B = _basis(degree_source)
    return np.array([[sum(float(c) * x[0] ** e[0] * x[1] ** e[1] * x[2] ** e[2] for e, c in phi.items())
                      for phi in B] for x in X])


def interpolate_same_map(u0, dofs0, dofs1, im, n_target_blocks, bs=1, u1=None):
    """The reference algorithm (interpolate_same_map, CUDAInterpolate.cu):
    gather each cell's source values X0 = u0[M0], X1 = IM X0, scatter
    u1[M1] = X1 with cells in order (a later cell overwrites a shared dof)."""
    u1 = np.zeros(n_target_blocks * bs) if u1 is None else u1.copy()
    d0, d1 = np.asarray(dofs0, dtype=np.int64), np.asarray(dofs1, dtype=np.int64)
    for q in range(bs):
        X1 = np.asarray(u0)[d0 * bs + q] @ np.asarray(im).T
        for c in range(len(d1)):
            u1[d1[c] * bs + q] = X1[c]
    return u1


# ---------------------------------------------------------------------------
# Jacobi-preconditioned CG (the reference hands A, b to PETSc KSP cg+jacobi:
# python/examples/poisson.py:116-125)
# ---------------------------------------------------------------------------

def pcg_jacobi(row_ptr, col, values, b, rtol=1e-8, max_iter=10000):
    import scipy.sparse as sp
    n = len(row_ptr) - 1
    A = sp.csr_matrix((values, col, row_ptr), shape=(n, n))
    dinv = 1.0 / A.diagonal()
    x = np.zeros(n)
    r = b - A @ x
    z = dinv * r
    p = z.copy()
    rz = r @ z
    b_norm = np.linalg.norm(b)
    it = 0
    while it < max_iter:
        if np.linalg.norm(r) <= rtol * b_norm:
            break
        Ap = A @ p
        alpha = rz / (p @ Ap)
        x += alpha * p
        r -= alpha * Ap
        z = dinv * r
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
        it += 1
    return x, it


# ---------------------------------------------------------------------------
# Problem builders for the benchmark configurations
# ---------------------------------------------------------------------------

def build_problem(kind: str, n: int, seed: int = 0):
    """Synthetic problem instances (seeded numpy inputs).

    kind: 'p1'   -- P1 Poisson, k=1, f = P1 interpolant of sin(pi x)sin(pi y)sin(pi z),
                    homogeneous Dirichlet on the whole boundary.
          'p2'   -- P2 Poisson, k = exp(N(0,1)) per vertex (P1 field), f ~ U[-1,1]
                    per cell (DG0), g = x + y + z on the boundary.
          'vp2'  -- vector P2 elasticity, lam ~ U[0.5,2], mu ~ U[0.2,1] per cell,
                    vertices jittered +-0.2h, body force (0,0,-1), u = 0 on the boundary.
          'p1k'  -- P1 Poisson with DG0 k log-uniform in [1e-2,1e2] per cell.
          'p3'   -- equispaced P3 Poisson, k = exp(N(0,1)) and f ~ U[-1,1] per cell
                    (DG0), g = x + y + z on the boundary.
    """
    rng = np.random.default_rng(seed)
    P = {"kind": kind, "n": n}
    if kind == "vp2":
        coords, cells = unit_cube_tet_mesh(n, jitter=0.2, seed=seed)
    else:
        coords, cells = unit_cube_tet_mesh(n)
    P["coords"], P["cells"] = coords, cells
    C = len(cells)
    if kind in ("p1", "p1k"):
        dofs = cells.copy()
        ndof = len(coords)
        grid = vertex_grid_index(n)
        bnd = boundary_dofs_from_grid(grid, n)
        X = coords
        P.update(dofs=dofs, ndof=ndof, bs=1, degree=1, bc_dofs=bnd)
        if kind == "p1":
            f = np.sin(np.pi * X[:, 0]) * np.sin(np.pi * X[:, 1]) * np.sin(np.pi * X[:, 2])
            P.update(k=None, f=f, g=np.zeros(ndof))
        else:
            k = np.exp(rng.uniform(np.log(1e-2), np.log(1e2), size=C))
            f = np.ones(ndof)
            P.update(k=k, f=f, g=np.zeros(ndof))
    elif kind == "p2":
        dofs, ndof, grid = p2_dofmap(n, cells)
        X = dof_coordinates(coords, cells, dofs, ndof, 2)
        bnd = boundary_dofs_from_grid(grid, 2 * n)
        kv = np.exp(rng.standard_normal(len(coords)))
        f = rng.uniform(-1.0, 1.0, size=C)
        g = X.sum(axis=1)
        P.update(dofs=dofs, ndof=ndof, bs=1, degree=2, bc_dofs=bnd, k=kv, f=f, g=g)
    elif kind == "p3":
        dofs, ndof, grid = p3_dofmap(n, cells)
        X = dof_coordinates(coords, cells, dofs, ndof, 3)
        bnd = boundary_dofs_from_grid(grid, 3 * n)
        k = np.exp(rng.standard_normal(C))
        f = rng.uniform(-1.0, 1.0, size=C)
        P.update(dofs=dofs, ndof=ndof, bs=1, degree=3, bc_dofs=bnd, k=k, f=f, g=X.sum(axis=1))
    elif kind == "vp2":
        dofs, ndof, grid = p2_dofmap(n, cells)
        bnd_nodes = boundary_dofs_from_grid(grid, 2 * n)
        bnd = (bnd_nodes[:, None] * 3 + np.arange(3)).ravel().astype(np.int32)
        lam = rng.uniform(0.5, 2.0, size=C)
        mu = rng.uniform(0.2, 1.0, size=C)
        f3 = np.tile(np.array([0.0, 0.0, -1.0]), (C, 1))
        P.update(dofs=dofs, ndof=ndof, bs=3, degree=2, bc_dofs=bnd, lam=lam, mu=mu, f=f3,
                 g=np.zeros(3 * ndof))
    else:
        raise ValueError(kind)
    return P


def element_matrices(P):
    kind = P["kind"]
    if kind in ("p1", "p1k"):
        return p1_stiffness(P["coords"], P["cells"], P["k"])
    if kind == "p2":
        return p2_stiffness(P["coords"], P["cells"], P["k"][P["cells"]])
    if kind == "p3":
        return p3_stiffness(P["coords"], P["cells"], P["k"])
    if kind == "vp2":
        return p2_elasticity(P["coords"], P["cells"], P["lam"], P["mu"])
    raise ValueError(kind)


def element_vectors(P):
    kind = P["kind"]
    if kind in ("p1", "p1k"):
        return p1_load_p1f(P["coords"], P["cells"], P["f"])
    if kind == "p2":
        return p2_load_dg0(P["coords"], P["cells"], P["f"])
    if kind == "p3":
        return p3_load_dg0(P["coords"], P["cells"], P["f"])
    if kind == "vp2":
        return p2_vector_load_dg0(P["coords"], P["cells"], P["f"])
    raise ValueError(kind)


def solve_system(P):
    """Full oracle pipeline: A with BCs, b = assemble + lifting + set_bc.
    Returns dict(row_ptr, col, A, b, markers, A_bound, b_bound), the last two
    the per-entry parity bounds (matrix_bound, vector_bound + lifting_bound,
    0 on the set_bc rows)."""
    bs = P["bs"]
    dofs = P["dofs"]
    nscal = P["ndof"] * bs
    row_ptr, col = sparsity(dofs, dofs, P["ndof"], bs, bs)
    markers = np.zeros(nscal, dtype=np.uint8)
    markers[P["bc_dofs"]] = 1
    Ae = element_matrices(P)
    A = assemble_matrix(Ae, dofs, dofs, row_ptr, col, bs, bs, markers, markers, 1.0, P["bc_dofs"])
    be = element_vectors(P)
    b = assemble_vector(be, dofs, nscal, bs)
    b = apply_lifting(b, Ae, dofs, dofs, markers, P["g"], None, 1.0, bs, bs)
    b = set_bc(b, P["bc_dofs"], P["g"])
    A_bound = matrix_bound(Ae, dofs, dofs, row_ptr, col, bs, bs, markers, markers)
    b_bound = vector_bound(be, dofs, nscal, bs) + lifting_bound(nscal, Ae, dofs, dofs, markers, P["g"], None,
                                                                1.0, bs, bs)
    b_bound[np.asarray(P["bc_dofs"])] = 0.0
    return {"row_ptr": row_ptr, "col": col, "A": A, "b": b, "markers": markers, "A_bound": A_bound,
            "b_bound": b_bound}


def nnz_formula(kind: str, n: int) -> int:
    """Closed-form nnz for the unit-cube meshes."""
    V = (n + 1) ** 3
    E = 3 * n * (n + 1) ** 2 + 3 * n * n * (n + 1) + n ** 3
    if kind in ("p1", "p1k"):
        return V + 2 * E
    if kind == "p3":
        # cubic in n through the counts at n = 1..4 (1816, 12415, 39664,
        # 91429); row widths are fixed per node class away from the boundary
        return 1311 * n ** 3 + 459 * n ** 2 + 45 * n + 1
    p2 = 230 * n ** 3 + 138 * n ** 2 + 24 * n + 1
    return p2 if kind == "p2" else 9 * p2


# ---------------------------------------------------------------------------
# Quadrature-evaluated forms: the oracle of forms given as FFCx
# tabulate_tensor bodies (python/cudolfinx/jit.py:15-114 feeds the reference
# such bodies; FFCx integrates with a basix quadrature rule).  Everything here
# is evaluated per cell in physical coordinates with numpy, independently of
# any generated code: the rule and the points are the only shared input.
# ---------------------------------------------------------------------------
REF_TET = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


def _gauss01(n):
    t, w = np.polynomial.legendre.leggauss(n)
    return 0.5 * (t + 1.0), 0.5 * w


@lru_cache(maxsize=None)
def tet_rule(n: int):
    """Collapsed Gauss-Legendre rule on the reference tetrahedron: n^3 points,
    x = a(1-b)(1-c), y = b(1-c), z = c; exact for total degree <= 2n - 3."""
    t, w = _gauss01(n)
    a, b, c = np.meshgrid(t, t, t, indexing="ij")
    wa, wb, wc = np.meshgrid(w, w, w, indexing="ij")
    X = np.stack([a * (1 - b) * (1 - c), b * (1 - c), c], axis=-1).reshape(-1, 3)
    W = (wa * wb * wc * (1 - b) * (1 - c) ** 2).ravel()
    return X, W


@lru_cache(maxsize=None)
def tri_rule(n: int):
    """Collapsed Gauss-Legendre rule on the reference triangle: n^2 points,
    x = a(1-b), y = b; exact for total degree <= 2n - 2."""
    t, w = _gauss01(n)
    a, b = np.meshgrid(t, t, indexing="ij")
    wa, wb = np.meshgrid(w, w, indexing="ij")
    return np.stack([a * (1 - b), b], axis=-1).reshape(-1, 2), (wa * wb * (1 - b)).ravel()


def lagrange_tables(degree: int, X):
    """Values [N, k] and reference gradients [N, k, 3] of the Lagrange basis
    (degree 0: the constant; 1, 2, 3: the basix-ordered bases above) at the
    reference points X [N, 3]."""
    X = np.asarray(X, dtype=float)
    if degree == 0:
        return np.ones((len(X), 1)), np.zeros((len(X), 1, 3))
    phi = _basis(degree)
    xs, ys, zs = X[:, 0], X[:, 1], X[:, 2]

    def ev(p):
        out = np.zeros(len(X))
        for (a, b, c), v in p.items():
            out += float(v) * xs ** a * ys ** b * zs ** c
        return out

    V = np.stack([ev(p) for p in phi], axis=1)
    D = np.stack([np.stack([ev(_pdiff(p, ax)) for ax in range(3)], axis=-1) for p in phi], axis=1)
    return V, D


def facet_points(f: int, P2):
    """Reference-tetrahedron points of the reference-triangle points P2 [N, 2]
    on local facet f: v0 + x (v1 - v0) + y (v2 - v0), (v0, v1, v2) the facet's
    vertices in TET_FACETS order."""
    v = REF_TET[list(TET_FACETS[f])]
    P2 = np.asarray(P2, dtype=float)
    return v[0] + P2[:, :1] * (v[1] - v[0]) + P2[:, 1:2] * (v[2] - v[0])


def facet_permutation(global_vertices) -> int:
    """Quadrature permutation code of a triangle facet: 2*rot + ref, rot the
    position (in the cell's local facet order) of its lowest-numbered global
    vertex, ref = 1 when the vertex after it (cyclically) is numbered above
    the vertex before it."""
    gv = list(global_vertices)
    rot = 0
    for t in (1, 2):
        if gv[t] < gv[rot]:
            rot = t
    pre, post = gv[(rot + 2) % 3], gv[(rot + 1) % 3]
    return 2 * rot + (1 if post > pre else 0)


def permute_facet_points(P2, code: int):
    """Points of the rule for facet permutation `code`: reflected (x, y) -> (y, x)
    when ref, then rotated rot times by (x, y) -> (1 - x - y, x).  With the
    codes of facet_permutation the two cells of an interior facet then see
    the same physical points (checked in tests/test_oracle.py)."""
    P = np.asarray(P2, dtype=float).copy()
    rot, ref = code // 2, code % 2
    if ref:
        P = P[:, ::-1].copy()
    for _ in range(rot):
        P = np.stack([1.0 - P[:, 0] - P[:, 1], P[:, 0]], axis=1)
    return P


def _jacobians(coords, cells):
    x = coords[cells]  # [C, 4, 3]
    J = np.transpose(x[:, 1:] - x[:, :1], (0, 2, 1))  # J[c, r, k] = x_{k+1, r} - x_{0, r}
    return x, J, np.linalg.det(J), np.linalg.inv(J)


def _phys_grad(K, D):
    """grad_x phi = K^T grad_X phi: K [C, 3, 3], D [..., k, 3] -> [C, ..., k, 3]."""
    return np.einsum("cba,...ib->c...ia", K, D)


def quad_cell_forms(coords, cells, u, kappa, n=4):
    """The nonlinear P1 test forms, with u and kappa P1 fields given per cell
    [C, 4] (vertex values), integrated by tet_rule(n):
      residual  R_i  = int exp(u) kappa phi_i + grad u . grad phi_i,
      jacobian  J_ij = int exp(u) kappa phi_j phi_i + grad phi_j . grad phi_i,
      functional     = int exp(u) kappa.
    Returns (R [C, 4], J [C, 4, 4], M [C])."""
    X, w = tet_rule(n)
    V, D = lagrange_tables(1, X)
    _, _, det, K = _jacobians(coords, cells)
    G = _phys_grad(K, D[0])  # P1 gradients are constant: [C, 4, 3]
    uq = u @ V.T  # [C, N]
    kq = kappa @ V.T
    gu = np.einsum("ci,cia->ca", u, G)
    dx = np.abs(det)[:, None] * w[None, :]  # [C, N]
    e = np.exp(uq) * kq * dx
    R = e @ V + (dx.sum(axis=1) * np.einsum("ca,cia->ci", gu, G).T).T
    Jm = np.einsum("cq,qi,qj->cij", e, V, V) + dx.sum(axis=1)[:, None, None] * np.einsum("cia,cja->cij", G, G)
    return R, Jm, e.sum(axis=1)


def quad_cell_matrix(coords, cells, test_degree, trial_degree, integrand, n=4):
    """[C, k0, k1] of int integrand(V0, G0, V1, G1) dx by tet_rule(n), with
    V [N, k] values and G [C, N, k, 3] physical gradients of the test / trial
    bases; integrand returns [C, N, k0, k1]."""
    X, w = tet_rule(n)
    V0, D0 = lagrange_tables(test_degree, X)
    V1, D1 = lagrange_tables(trial_degree, X)
    _, _, det, K = _jacobians(coords, cells)
    G0, G1 = _phys_grad(K, D0), _phys_grad(K, D1)
    f = integrand(V0, G0, V1, G1)
    return np.einsum("cqij,cq->cij", f, np.abs(det)[:, None] * w[None, :])


def exterior_facet_forms(coords, cells, facets, u, kappa, n=3):
    """The reference's exterior-facet test forms on P1 (u, kappa P1 given per
    cell [C, 4]) over facets [F, 2] (cell, local facet), tri_rule(n):
      residual R_i  = int_F u kappa phi_i (grad u . n) ds,
      jacobian J_ij = int_F (phi_j kappa phi_i (grad u . n) + u kappa phi_i (grad phi_j . n)) ds,
    n the outward unit normal.  Returns (R [F, 4], J [F, 4, 4])."""
    P2, w = tri_rule(n)
    c, lf = facets[:, 0], facets[:, 1]
    x, _, _, K = _jacobians(coords, cells)
    R = np.zeros((len(facets), 4))
    Jm = np.zeros((len(facets), 4, 4))
    D = lagrange_tables(1, REF_TET[:1])[1][0]  # [4, 3]
    for f in range(4):
        sel = np.nonzero(lf == f)[0]
        if not len(sel):
            continue
        V = lagrange_tables(1, facet_points(f, P2))[0]  # [N, 4]
        xc = x[c[sel]]
        fv = xc[:, list(TET_FACETS[f])]  # [S, 3, 3]
        cr = np.cross(fv[:, 1] - fv[:, 0], fv[:, 2] - fv[:, 0])
        area2 = np.linalg.norm(cr, axis=1)
        nrm = cr / area2[:, None]
        opp = xc[:, f]  # the vertex off the facet: the normal points away from it
        sgn = np.sign(np.einsum("sa,sa->s", nrm, fv[:, 0] - opp))
        nrm = nrm * sgn[:, None]
        G = _phys_grad(K[c[sel]], D)  # [S, 4, 3]
        us, ks = u[c[sel]], kappa[c[sel]]
        uq, kq = us @ V.T, ks @ V.T  # [S, N]
        gun = np.einsum("si,sia,sa->s", us, G, nrm)  # grad u . n, constant on P1
        gpn = np.einsum("sja,sa->sj", G, nrm)
        ds = area2[:, None] * w[None, :]
        R[sel] = np.einsum("sq,qi->si", uq * kq * gun[:, None] * ds, V)
        Jm[sel] = (np.einsum("sq,qi,qj->sij", kq * gun[:, None] * ds, V, V)
                   + np.einsum("sq,qi,sj->sij", uq * kq * ds, V, gpn))
    return R, Jm


def interior_facet_points(coords, cells, quads, n=3):
    """Physical points [F, N, 3] and measures w*|J_F| [F, N] of tri_rule(n)
    on every interior facet, placed as cell 0 sees them (its facet
    permutation applied), plus the reference points of cell 0 [F, N, 3]."""
    P2, w = tri_rule(n)
    quads = np.asarray(quads)
    c0, f0 = quads[:, 0], quads[:, 1]
    x = coords[cells[c0]]
    Xref = np.zeros((len(quads), len(w), 3))
    for e in range(len(quads)):
        gv = cells[c0[e]][list(TET_FACETS[f0[e]])]
        Xref[e] = facet_points(f0[e], permute_facet_points(P2, facet_permutation(gv)))
    J = np.transpose(x[:, 1:] - x[:, :1], (0, 2, 1))
    Xphys = x[:, :1] + np.einsum("frk,fqk->fqr", J, Xref)
    fv = x[np.arange(len(quads))[:, None], np.array(TET_FACETS)[f0]]
    area2 = np.linalg.norm(np.cross(fv[:, 1] - fv[:, 0], fv[:, 2] - fv[:, 0]), axis=1)
    return Xphys, area2[:, None] * w[None, :], Xref


def interior_facet_forms(coords, cells, quads, u_dg1, kappa_p1, p1_cells, alpha, n=3):
    """Interior-facet test forms of DG1 (u, the test and trial spaces) with a P1
    kappa, by tri_rule(n) at points located on each side independently
    (barycentric coordinates of the physical points):
      residual   R  [F, 8] = int avg(v) avg(kappa) avg(u^2) dS,
      jacobian   Jm [F, 8, 8] = int avg(v) avg(kappa) avg(2 u du) dS,
      functional M  [F]    = int avg(u^2) avg(kappa) dS,
      SIPG       S  [F, 8, 8] = int (-avg(grad du . n) jump(v) - jump(du) avg(grad v . n)
                                     + alpha jump(du) jump(v)) dS,
    macro dofs cell 0's then cell 1's, jump(w) = w(cell 0) - w(cell 1), n the
    unit normal pointing out of cell 0; u_dg1 [C, 4] per cell, kappa_p1
    vertex values through p1_cells."""
    quads = np.asarray(quads)
    Xp, dS, _ = interior_facet_points(coords, cells, quads, n)
    c0, f0, c1 = quads[:, 0], quads[:, 1], quads[:, 2]
    L0 = _barycentric(coords, cells, c0, Xp)  # [F, N, 4]: the P1 / DG1 basis values
    L1 = _barycentric(coords, cells, c1, Xp)
    _, _, _, K = _jacobians(coords, cells)
    D = lagrange_tables(1, REF_TET[:1])[1][0]
    G0, G1 = _phys_grad(K[c0], D), _phys_grad(K[c1], D)  # [F, 4, 3]
    x0 = coords[cells[c0]]
    fv = x0[np.arange(len(quads))[:, None], np.array(TET_FACETS)[f0]]
    cr = np.cross(fv[:, 1] - fv[:, 0], fv[:, 2] - fv[:, 0])
    nrm = cr / np.linalg.norm(cr, axis=1)[:, None]
    opp = x0[np.arange(len(quads)), f0]
    nrm = nrm * np.sign(np.einsum("fa,fa->f", nrm, fv[:, 0] - opp))[:, None]
    kv = np.asarray(kappa_p1)
    k0 = np.einsum("fqi,fi->fq", L0, kv[p1_cells[c0]])
    k1 = np.einsum("fqi,fi->fq", L1, kv[p1_cells[c1]])
    u0 = np.einsum("fqi,fi->fq", L0, u_dg1[c0])
    u1 = np.einsum("fqi,fi->fq", L1, u_dg1[c1])
    kav = 0.5 * (k0 + k1)
    u2av = 0.5 * (u0 ** 2 + u1 ** 2)
    Vm = np.concatenate([0.5 * L0, 0.5 * L1], axis=2)  # avg(v) of the macro basis
    R = np.einsum("fq,fqi->fi", dS * kav * u2av, Vm)
    dU = np.concatenate([0.5 * 2 * u0[:, :, None] * L0, 0.5 * 2 * u1[:, :, None] * L1], axis=2)  # avg(2 u du)
    Jm = np.einsum("fq,fqi,fqj->fij", dS * kav, Vm, dU)
    M = np.einsum("fq->f", dS * u2av * kav)
    jump = np.concatenate([L0, -L1], axis=2)  # [F, N, 8]
    gn = np.concatenate([np.einsum("fia,fa->fi", G0, nrm), np.einsum("fia,fa->fi", G1, nrm)], axis=1)  # [F, 8]
    avg_gn = 0.5 * gn  # avg(grad w . n) of each macro basis function (constant per facet on P1)
    S = (-np.einsum("fq,fj,fqi->fij", dS, avg_gn, jump) - np.einsum("fq,fqj,fi->fij", dS, jump, avg_gn)
         + alpha * np.einsum("fq,fqi,fqj->fij", dS, jump, jump))
    return R, Jm, M, S
