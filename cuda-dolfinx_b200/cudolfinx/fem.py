"""Host-side stand-ins for the DOLFINx objects the cudolfinx API consumes.

The reference takes DOLFINx meshes, function spaces, Functions, DirichletBCs
and UFL forms (python/cudolfinx/assemble.py, form.py, bcs.py).  DOLFINx is not
part of this engine, so this module provides the minimal equivalents the
assembly path needs, with DOLFINx's data layout:

* ``create_unit_cube(n)``  -- the topology of ``dolfinx.mesh.create_box`` with
  ``CellType.tetrahedron``: n^3 hexes, 6 tets each, sharing the v0-v7 diagonal
  (python/examples/poisson.py:34-40); vertex (ix,iy,iz) -> iz(n+1)^2 + iy(n+1) + ix.
* ``functionspace(mesh, ("P", 1|2[, (3,)]))`` -- Lagrange dofmaps, local dof
  order = basix (4 vertices, then edges (2,3),(1,3),(1,2),(0,3),(0,2),(0,1));
  blocked spaces keep one block dof per node (bs = 3), as DOLFINx does.
* ``Function``, ``dirichletbc``, ``locate_boundary_dofs``.
* form constructors ``stiffness``, ``elasticity``, ``load`` returning
  ``FormSpec`` objects that ``cudolfinx.form`` compiles (they stand where the
  UFL forms stand in the reference).

P2 numbering: every point of the doubled (2n+1)^3 grid is a P2 node on this
mesh (vertices: all coordinates even; axis edges: one odd; the face diagonals
v0-v3, v0-v5, v0-v6 and their translates: two odd; body diagonals: three
odd), so dof = (Z*(2n+1) + Y)*(2n+1) + X, which keeps neighbouring nodes close
in memory.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence, Union

import numpy as np

TET_EDGES = ((2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1))

# barycentric weights (in thirds) of the 20 equispaced P3 nodes in basix's
# local order: vertices; per edge (a, b) the point nearer a, then the one
# nearer b; per face f (opposite vertex f) its centroid
_P3_WEIGHTS = np.array(
    [[3 if q == v else 0 for q in range(4)] for v in range(4)]
    + [w for a, b in TET_EDGES
       for w in ([2 if q == a else (1 if q == b else 0) for q in range(4)],
                 [1 if q == a else (2 if q == b else 0) for q in range(4)])]
    + [[0 if q == f else 1 for q in range(4)] for f in range(4)], dtype=np.int64)


class Mesh:
    """Affine tetrahedral mesh: coordinates (N,3) float64 and cells (C,4) int32."""

    def __init__(self, coords: np.ndarray, cells: np.ndarray, grid_n: Optional[int] = None):
        self.geometry_x = np.ascontiguousarray(coords, dtype=np.float64)
        self.cells = np.ascontiguousarray(cells, dtype=np.int32)
        self.grid_n = grid_n  # structured unit-cube resolution, if any
        self._uid = id(self)

    @property
    def num_cells(self) -> int:
        return len(self.cells)

    @property
    def num_vertices(self) -> int:
        return len(self.geometry_x)


def create_unit_cube(n: int, jitter: float = 0.0, seed: int = 0) -> Mesh:
    """Unit cube, n^3 hexes x 6 tets.  ``jitter`` moves every vertex by
    U[-jitter*h, jitter*h] per coordinate except normal to the boundary planes
    it lies on (the domain stays the unit cube)."""
    n1 = n + 1
    ix = np.arange(n1 ** 3) % n1
    iy = (np.arange(n1 ** 3) // n1) % n1
    iz = np.arange(n1 ** 3) // (n1 * n1)
    idx = np.stack([ix, iy, iz], axis=1)
    coords = idx / float(n)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-jitter / n, jitter / n, size=coords.shape)
        d[(idx == 0) | (idx == n)] = 0.0
        coords = coords + d
    hz, hy, hx = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    v0 = (hz * n1 * n1 + hy * n1 + hx).ravel()
    s_x, s_y, s_z = 1, n1, n1 * n1
    v1, v2, v3 = v0 + s_x, v0 + s_y, v0 + s_x + s_y
    v4, v5, v6, v7 = v0 + s_z, v1 + s_z, v2 + s_z, v3 + s_z
    cells = np.stack([
        np.stack([v0, v1, v3, v7], 1), np.stack([v0, v1, v7, v5], 1), np.stack([v0, v5, v7, v4], 1),
        np.stack([v0, v3, v2, v7], 1), np.stack([v0, v6, v4, v7], 1), np.stack([v0, v2, v6, v7], 1),
    ], axis=1).reshape(-1, 4)
    return Mesh(coords, cells.astype(np.int32), grid_n=n)


class FunctionSpace:
    """Lagrange space of degree 1, 2 or 3 (scalar; degree 2 also as a
    3-vector) on a Mesh.  Degree 3 uses equispaced points (basix's
    "equispaced" Lagrange variant)."""

    def __init__(self, mesh: Mesh, element):
        family, degree = element[0], int(element[1])
        shape = tuple(element[2]) if len(element) > 2 else ()
        if family not in ("P", "Lagrange", "CG", "DG"):
            raise ValueError(f"unsupported family {family}")
        self.mesh = mesh
        self.family = "DG" if family == "DG" else "P"
        self.degree = degree
        self.bs = 1 if shape == () else int(np.prod(shape))
        if self.bs not in (1, 3):
            raise ValueError("value shape must be () or (3,)")
        if self.family == "DG":
            if degree not in (0, 1) or self.bs != 1 and degree != 0:
                raise ValueError("DG0 (scalar or vector) and scalar DG1 are supported")
            # discontinuous: every cell owns its dofs (DG1: one per vertex, in
            # the cell's vertex order)
            k = 1 if degree == 0 else 4
            self.dofs = np.arange(mesh.num_cells * k, dtype=np.int32).reshape(-1, k)
            self.num_nodes = mesh.num_cells * k
            self._node_x = None
            self._grid = None
        elif degree == 1:
            self.dofs = mesh.cells.copy()
            self.num_nodes = mesh.num_vertices
            self._grid = None
        elif degree == 2:
            self._build_p2()
        elif degree == 3:
            if self.bs != 1:
                raise ValueError("degree 3 is offered for scalar spaces")
            self._build_p3()
        else:
            raise ValueError("degree must be 1, 2 or 3")
        self._uid = id(self)

    def _build_p2(self):
        m = self.mesh
        if m.grid_n is None:
            raise ValueError("P2 spaces are built for structured unit-cube meshes")
        n = m.grid_n
        n1, M = n + 1, 2 * n + 1
        v = m.cells.astype(np.int64)
        g = np.stack([v % n1, (v // n1) % n1, v // (n1 * n1)], axis=-1)  # [C,4,3]
        pts = [2 * g[:, a] for a in range(4)] + [g[:, a] + g[:, b] for a, b in TET_EDGES]
        P = np.stack(pts, axis=1)
        self.dofs = ((P[..., 2] * M + P[..., 1]) * M + P[..., 0]).astype(np.int32)
        self.num_nodes = M ** 3
        self._grid = (n, M)

    def _build_p3(self):
        # every point of the tripled (3n+1)^3 grid is a P3 node of this mesh
        # (each Kuhn tet's 20 nodes are grid points, and the tets cover every
        # point), numbered like the P2 nodes: dof = (Z*(3n+1) + Y)*(3n+1) + X
        m = self.mesh
        if m.grid_n is None:
            raise ValueError("P3 spaces are built for structured unit-cube meshes")
        n = m.grid_n
        n1, M = n + 1, 3 * n + 1
        v = m.cells.astype(np.int64)
        g = np.stack([v % n1, (v // n1) % n1, v // (n1 * n1)], axis=-1)  # [C,4,3]
        P = np.einsum("lv,cvd->cld", _P3_WEIGHTS, g)  # tripled-grid coordinates [C,20,3]
        self.dofs = ((P[..., 2] * M + P[..., 1]) * M + P[..., 0]).astype(np.int32)
        self.num_nodes = M ** 3
        self._grid = (n, M)

    # --- layout ------------------------------------------------------------
    @property
    def num_dofs(self) -> int:
        """Scalar (unrolled) dofs."""
        return self.num_nodes * self.bs

    @property
    def dofs_per_cell(self) -> int:
        return self.dofs.shape[1]

    def tabulate_dof_coordinates(self) -> np.ndarray:
        """(num_nodes, 3) physical node coordinates (affine cells)."""
        m = self.mesh
        X = np.zeros((self.num_nodes, 3))
        cx = m.geometry_x[m.cells]
        if self.family == "DG":
            return cx.mean(axis=1) if self.degree == 0 else cx.reshape(-1, 3).copy()
        if self.degree == 1:
            X[self.dofs.ravel()] = m.geometry_x[m.cells.ravel()]
            return X
        if self.degree == 3:
            P = np.einsum("lv,cvd->cld", _P3_WEIGHTS / 3.0, cx)
            X[self.dofs.ravel()] = P.reshape(-1, 3)
            return X
        pts = [cx[:, a] for a in range(4)] + [0.5 * (cx[:, a] + cx[:, b]) for a, b in TET_EDGES]
        X[self.dofs.ravel()] = np.stack(pts, axis=1).reshape(-1, 3)
        return X

    def boundary_nodes(self) -> np.ndarray:
        """Nodes on the boundary of the unit cube (exact, from grid indices)."""
        m = self.mesh
        if m.grid_n is None:
            raise ValueError("boundary location needs a structured unit-cube mesh")
        n = m.grid_n
        ext = self.degree * n
        N = ext + 1
        k = np.arange(N ** 3)
        ijk = np.stack([k % N, (k // N) % N, k // (N * N)], axis=1)
        return np.nonzero(np.any((ijk == 0) | (ijk == ext), axis=1))[0].astype(np.int32)

    def contains(self, other: "FunctionSpace") -> bool:
        return other is self


def reference_nodes(V: FunctionSpace) -> np.ndarray:
    """Reference coordinates [k, 3] of the element's nodes in local order
    (DG0: the centroid)."""
    if V.family == "DG" and V.degree == 0:
        return np.full((1, 3), 0.25)
    if V.degree == 1:
        W = np.eye(4)
    elif V.degree == 2:
        W = np.array([np.eye(4)[v] for v in range(4)] + [0.5 * (np.eye(4)[a] + np.eye(4)[b]) for a, b in TET_EDGES])
    else:
        W = _P3_WEIGHTS / 3.0
    return W[:, 1:].copy()  # (x, y, z) = (l1, l2, l3)


def lagrange_basis(V: FunctionSpace, X: np.ndarray) -> np.ndarray:
    """Values [npts, k] of the element's basis functions at reference points X
    (barycentric formulas of the equispaced Lagrange elements, basix local order)."""
    X = np.atleast_2d(np.asarray(X, dtype=np.float64))
    lam = np.column_stack([1.0 - X.sum(axis=1), X[:, 0], X[:, 1], X[:, 2]])
    if V.family == "DG" and V.degree == 0:
        return np.ones((len(X), 1))
    if V.degree == 1:
        return lam
    if V.degree == 2:
        vert = [lam[:, v] * (2 * lam[:, v] - 1) for v in range(4)]
        edge = [4 * lam[:, a] * lam[:, b] for a, b in TET_EDGES]
        return np.column_stack(vert + edge)
    vert = [0.5 * lam[:, v] * (3 * lam[:, v] - 1) * (3 * lam[:, v] - 2) for v in range(4)]
    edge = []
    for a, b in TET_EDGES:
        edge.append(4.5 * lam[:, a] * lam[:, b] * (3 * lam[:, a] - 1))
        edge.append(4.5 * lam[:, a] * lam[:, b] * (3 * lam[:, b] - 1))
    face = [27 * np.prod(lam[:, [q for q in range(4) if q != f]], axis=1) for f in range(4)]
    return np.column_stack(vert + edge + face)


def interpolation_matrix(V: FunctionSpace, V0: FunctionSpace) -> np.ndarray:
    """Interpolation operator [k, k0] from V0 into V on the same reference map:
    V's nodes evaluated in V0's basis (create_interpolation_operator of
    Lagrange elements)."""
    return np.ascontiguousarray(lagrange_basis(V0, reference_nodes(V)))


def functionspace(mesh: Mesh, element) -> FunctionSpace:
    return FunctionSpace(mesh, element)


class Function:
    """Finite-element function: host values ``x.array`` (scalar dofs)."""

    class _Vec:
        def __init__(self, n):
            self.array = np.zeros(n)

    def __init__(self, V: FunctionSpace, values: Optional[np.ndarray] = None):
        self.function_space = V
        self.x = Function._Vec(V.num_dofs)
        if values is not None:
            self.x.array[:] = values

    def interpolate(self, f: Callable[[np.ndarray], np.ndarray]):
        """Nodal interpolation: f receives x of shape (3, num_nodes)."""
        X = self.function_space.tabulate_dof_coordinates().T
        vals = np.asarray(f(X), dtype=np.float64)
        if self.function_space.bs == 1:
            self.x.array[:] = vals.reshape(-1)
        else:
            self.x.array[:] = vals.reshape(self.function_space.bs, -1).T.reshape(-1)


def locate_boundary_dofs(V: FunctionSpace) -> np.ndarray:
    """Scalar dofs on the boundary facets (blocked: every component)."""
    nodes = V.boundary_nodes()
    if V.bs == 1:
        return nodes
    return (nodes[:, None] * V.bs + np.arange(V.bs)).ravel().astype(np.int32)


class DirichletBC:
    """u = g on ``dofs`` (scalar dofs of V); g is a Function on V or a float."""

    def __init__(self, value: Union[Function, float], dofs: np.ndarray, V: Optional[FunctionSpace] = None):
        if isinstance(value, Function):
            V = value.function_space if V is None else V
        if V is None:
            raise ValueError("a constant BC value needs the function space V")
        self.function_space = V
        self.value = value
        self.dofs = np.ascontiguousarray(np.unique(np.asarray(dofs, dtype=np.int32)))

    def values(self) -> np.ndarray:
        g = np.zeros(self.function_space.num_dofs)
        if isinstance(self.value, Function):
            g[self.dofs] = self.value.x.array[self.dofs]
        else:
            g[self.dofs] = float(self.value)
        return g


def dirichletbc(value, dofs, V: Optional[FunctionSpace] = None) -> DirichletBC:
    return DirichletBC(value, dofs, V)


Coefficient = Union[Function, float, Sequence[float], np.ndarray]


@dataclass
class FormSpec:
    """A built-in variational form (stands where a UFL form stands)."""
    kind: str                      # 'P1_STIFFNESS', 'P2_STIFFNESS', 'VP2_ELASTICITY', '*_LOAD'
    V: FunctionSpace
    coefficients: list = field(default_factory=list)
    rank: int = 2
    precision: str = "fp64"
    facets: Optional[np.ndarray] = None  # exterior-facet forms: [F, 2] (cell, local facet)
    domain: Optional["Mesh"] = None      # functionals: the mesh (V may be None)
    W: Optional[FunctionSpace] = None    # bilinear forms: trial space when it is not V

    @property
    def function_spaces(self):
        if self.rank == 0:
            return []
        return [self.V, self.W if self.W is not None else self.V] if self.rank == 2 else [self.V]

    @property
    def mesh(self):
        return self.domain if self.domain is not None else self.V.mesh


@dataclass
class FFCxIntegral:
    """One integral of a form compiled by FFCx: the name and the body (the
    statements between the outer braces) of its tabulate_tensor_integral_*
    function, as python/cudolfinx/jit.py:15-59 extracts them from the
    generated C file, its integral type ("cell", "exterior_facet",
    "interior_facet") and, for facet integrals, the integration entities:
    [F, 2] (cell, local facet) or [F, 4] (cell0, facet0, cell1, facet1).
    Facet integrals without entities run over all exterior / interior facets
    of the mesh."""
    integral_type: str
    name: str
    body: str
    entities: Optional[np.ndarray] = None


@dataclass
class FFCxForm:
    """A variational form as FFCx compiles it (stands where a UFL form given to
    cudolfinx.form stands in the reference): its integrals, the argument
    spaces ([] functional, [V] linear, [V, U] bilinear: test, trial), the
    coefficients in FFCx's order (Functions; coefficient q has
    dofs_per_cell * bs values per cell) and the constants in the form's order
    (each a number or array, packed flat as DOLFINx pack_constants does).
    ``coefficient_sizes``, when given, are the values per cell the compiled
    form expects of each coefficient (the dimensions of the coefficient
    elements FFCx compiled it for); a coefficient whose space gives another
    number is rejected when the CUDA form is created."""
    integrals: list
    spaces: list
    coefficients: list = field(default_factory=list)
    constants: list = field(default_factory=list)
    domain: Optional["Mesh"] = None
    coefficient_sizes: Optional[list] = None

    @property
    def rank(self) -> int:
        return len(self.spaces)

    @property
    def function_spaces(self):
        return list(self.spaces)

    @property
    def mesh(self):
        if self.domain is not None:
            return self.domain
        if self.spaces:
            return self.spaces[0].mesh
        return self.coefficients[0].function_space.mesh

    def packed_constants(self) -> np.ndarray:
        if not self.constants:
            return np.zeros(0)
        return np.concatenate([np.atleast_1d(np.asarray(c, dtype=np.float64)).ravel() for c in self.constants])


def _trial(V: FunctionSpace, trial: Optional[FunctionSpace]) -> Optional[FunctionSpace]:
    if trial is None or trial is V:
        return None
    if (trial.mesh is not V.mesh or trial.family != V.family or trial.degree != V.degree or trial.bs != V.bs
            or not np.array_equal(trial.dofs, V.dofs)):
        raise ValueError("the trial space must be another copy of the test space's element on the same mesh")
    return trial


def stiffness(V: FunctionSpace, k: Coefficient = 1.0, precision: str = "fp64",
              trial: Optional[FunctionSpace] = None) -> FormSpec:
    """k * inner(grad(u), grad(v)) * dx on a scalar P1/P2/P3 space; u from
    ``trial`` (another space of the same element, e.g. the second field of a
    block system) when given."""
    if V.bs != 1 or V.family != "P":
        raise ValueError("stiffness needs a scalar Lagrange space")
    kind = {1: "P1_STIFFNESS", 2: "P2_STIFFNESS", 3: "P3_STIFFNESS"}[V.degree]
    return FormSpec(kind, V, [k], 2, precision, W=_trial(V, trial))


def mass(V: FunctionSpace, c: Coefficient = 1.0, trial: Optional[FunctionSpace] = None) -> FormSpec:
    """c * inner(u, v) * dx on a scalar P1/P2 or a vector P2 space; c constant,
    DG0 or a scalar P1 Function (FP64 element tensors; u from ``trial`` as for
    ``stiffness``).  Mass and stiffness (or elasticity) share their pattern, so
    M + dt K assembles into one matrix (the second call with zero=False)."""
    if V.family != "P" or not ((V.bs == 1 and V.degree in (1, 2)) or (V.bs == 3 and V.degree == 2)):
        raise ValueError("mass needs a scalar P1 / P2 or a vector P2 space")
    kind = "VP2_MASS" if V.bs == 3 else ("P1_MASS" if V.degree == 1 else "P2_MASS")
    return FormSpec(kind, V, [c], 2, "fp64", W=_trial(V, trial))


def elasticity(V: FunctionSpace, lam: Coefficient, mu: Coefficient, precision: str = "fp64",
               trial: Optional[FunctionSpace] = None) -> FormSpec:
    """2 mu eps(u):eps(v) + lam div(u) div(v) on a vector P2 space (u from
    ``trial`` when given, as for ``stiffness``)."""
    if V.bs != 3 or V.degree != 2:
        raise ValueError("elasticity needs a vector P2 space")
    return FormSpec("VP2_ELASTICITY", V, [lam, mu], 2, precision, W=_trial(V, trial))


# facet f of a tetrahedron is the one opposite vertex f (basix / DOLFINx)
_TET_FACETS = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])


def exterior_facets(mesh: "Mesh") -> np.ndarray:
    """(cell, local facet) pairs of the boundary facets -- the facets that
    belong to one cell only -- ordered by cell then local facet (the
    exterior-facet integration domain DOLFINx hands the reference,
    CUDAFormIntegral.cpp:361-447)."""
    cells = mesh.cells
    F = np.sort(cells[:, _TET_FACETS], axis=2).reshape(-1, 3)
    _, inv, cnt = np.unique(F, axis=0, return_inverse=True, return_counts=True)
    ext = np.nonzero(cnt[inv.ravel()] == 1)[0]
    return np.ascontiguousarray(np.stack([ext // 4, ext % 4], axis=1).astype(np.int32))


def facet_mass(V: FunctionSpace, alpha: Coefficient = 1.0, facets: Optional[np.ndarray] = None) -> FormSpec:
    """alpha * u * v * ds over exterior facets (Robin term) on scalar P1/P2;
    alpha constant or DG0 (the value of the facet's cell)."""
    if V.bs != 1 or V.family != "P" or V.degree not in (1, 2):
        raise ValueError("facet_mass needs a scalar P1 or P2 space")
    facets = exterior_facets(V.mesh) if facets is None else np.ascontiguousarray(facets, dtype=np.int32)
    return FormSpec("P1_FACET_MASS" if V.degree == 1 else "P2_FACET_MASS", V, [alpha], 2, "fp64", facets)


def facet_load(V: FunctionSpace, g: Coefficient, facets: Optional[np.ndarray] = None) -> FormSpec:
    """inner(g, v) * ds over exterior facets (Neumann / traction term) on P1,
    P2 or vector P2; g constant, DG0 or (scalar) P1."""
    if V.family != "P" or V.degree not in (1, 2):
        raise ValueError("facet_load needs a P1, P2 or vector-P2 space")
    facets = exterior_facets(V.mesh) if facets is None else np.ascontiguousarray(facets, dtype=np.int32)
    if V.bs == 3:
        kind = "VP2_FACET_LOAD"
    else:
        kind = "P1_FACET_LOAD" if V.degree == 1 else "P2_FACET_LOAD"
    return FormSpec(kind, V, [g], 1, "fp64", facets)


def integral(f: Coefficient, mesh: Optional["Mesh"] = None) -> FormSpec:
    """The functional int f dx; f constant (give the mesh), DG0 or P1."""
    mesh = mesh if mesh is not None else f.function_space.mesh
    return FormSpec("INTEGRAL", None, [f], 0, "fp64", None, mesh)


def energy(u: "Function", k: Coefficient = 1.0) -> FormSpec:
    """The functional int k |grad u|^2 dx for a scalar P1 or P2 Function u
    (k constant or DG0); equals u^T A u for the stiffness matrix A."""
    V = u.function_space
    if V.bs != 1 or V.family != "P" or V.degree not in (1, 2):
        raise ValueError("energy needs a scalar P1 or P2 Function")
    return FormSpec("P1_ENERGY" if V.degree == 1 else "P2_ENERGY", None, [k, u], 0, "fp64", None, V.mesh)


def facet_integral(g: Coefficient, mesh: "Mesh", facets: Optional[np.ndarray] = None) -> FormSpec:
    """The functional int g ds over exterior facets; g constant, DG0 or P1."""
    facets = exterior_facets(mesh) if facets is None else np.ascontiguousarray(facets, dtype=np.int32)
    return FormSpec("FACET_INTEGRAL", None, [g], 0, "fp64", facets, mesh)


def interior_facets(mesh: "Mesh") -> np.ndarray:
    """(cell0, local facet0, cell1, local facet1) of every facet shared by two
    cells, cell0 < cell1, ordered by the facet's sorted vertex triple (the
    interior-facet integration domain DOLFINx hands the reference,
    CUDAFormIntegral.cpp:451-522)."""
    F = np.sort(mesh.cells[:, _TET_FACETS], axis=2).reshape(-1, 3)
    _, inv, cnt = np.unique(F, axis=0, return_inverse=True, return_counts=True)
    inv = inv.ravel()
    order = np.argsort(inv, kind="stable")
    start = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    two = np.nonzero(cnt == 2)[0]
    e0, e1 = order[start[two]], order[start[two] + 1]
    return np.ascontiguousarray(np.stack([e0 // 4, e0 % 4, e1 // 4, e1 % 4], axis=1).astype(np.int32))


def _dg(V: FunctionSpace) -> int:
    if V.family != "DG" or V.bs != 1 or V.degree not in (0, 1):
        raise ValueError("interior-facet forms act on scalar DG0 / DG1 spaces")
    return V.degree


def jump_penalty(V: FunctionSpace, alpha: Coefficient = 1.0, facets: Optional[np.ndarray] = None) -> FormSpec:
    """alpha * jump(u) * jump(v) * dS over interior facets on DG0 / DG1
    (jump = value from cell0 minus value from cell1); alpha constant or DG0,
    averaged over the two cells of a facet."""
    kind = "DG0_JUMP" if _dg(V) == 0 else "DG1_JUMP"
    facets = interior_facets(V.mesh) if facets is None else np.ascontiguousarray(facets, dtype=np.int32)
    return FormSpec(kind, V, [alpha], 2, "fp64", facets)


def facet_average_load(V: FunctionSpace, g: Coefficient = 1.0, facets: Optional[np.ndarray] = None) -> FormSpec:
    """g * avg(v) * dS over interior facets on DG0 / DG1; g constant or DG0
    (averaged over the two cells)."""
    kind = "DG0_AVG_LOAD" if _dg(V) == 0 else "DG1_AVG_LOAD"
    facets = interior_facets(V.mesh) if facets is None else np.ascontiguousarray(facets, dtype=np.int32)
    return FormSpec(kind, V, [g], 1, "fp64", facets)


def jump_norm(u: "Function", facets: Optional[np.ndarray] = None) -> FormSpec:
    """The functional int jump(u)^2 dS over interior facets for a DG0, DG1 or
    P1 Function u (zero for a continuous u)."""
    V = u.function_space
    if V.bs != 1 or V.degree not in (0, 1) or (V.family == "P" and V.degree != 1):
        raise ValueError("jump_norm needs a scalar DG0, DG1 or P1 Function")
    facets = interior_facets(V.mesh) if facets is None else np.ascontiguousarray(facets, dtype=np.int32)
    return FormSpec("JUMP_NORM", None, [u], 0, "fp64", facets, V.mesh)


def load(V: FunctionSpace, f: Coefficient) -> FormSpec:
    """inner(f, v) * dx on P1 / P2 / P3 / vector P2."""
    if V.bs == 3:
        kind = "VP2_LOAD"
    else:
        kind = {1: "P1_LOAD", 2: "P2_LOAD", 3: "P3_LOAD"}[V.degree]
    return FormSpec(kind, V, [f], 1)
