"""Oracle pins (CPU): closed-form known answers, golden fixtures, C port vs numpy.

The reference ships no golden vectors, so the oracle is pinned to results
that follow from the mathematics alone, then frozen as fixtures.
"""
import glob
import os

import numpy as np
import pytest

from oracle import cfem
from oracle import fem_oracle as fo

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_TET = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
ONE_CELL = np.array([[0, 1, 2, 3]], dtype=np.int32)


def test_p1_reference_stiffness_known_answer():
    # classical P1 Laplacian on the unit reference tet: (1/6) [[3,-1,-1,-1],[-1,1,0,0],...]
    A = fo.p1_stiffness(REF_TET, ONE_CELL)[0] * 6
    expect = np.array([[3, -1, -1, -1], [-1, 1, 0, 0], [-1, 0, 1, 0], [-1, 0, 0, 1.0]])
    assert np.allclose(A, expect, atol=1e-15)


def test_basis_integrals_known_answer():
    # int phi = -|T|/20 (P2 vertex), |T|/5 (P2 edge), |T|/4 (P1), |T| = 1/6
    w2 = fo.ref_basis_integrals(2)
    assert np.allclose(w2[:4], -1.0 / 120) and np.allclose(w2[4:], 1.0 / 30)
    assert np.allclose(fo.ref_basis_integrals(1), 1.0 / 24)


def test_p2_reference_tensor_weights_sum_to_unweighted():
    # sum_m lambda_m = 1  =>  sum_m R[m] == R0
    assert np.allclose(fo.ref_grad_tensor(2, True).sum(axis=0), fo.ref_grad_tensor(2, False), atol=1e-15)


def _random_tet(rng):
    while True:
        x = rng.uniform(-1, 1, size=(4, 3))
        J = (x[1:] - x[0]).T
        if abs(np.linalg.det(J)) > 0.05:
            return x


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_stiffness_kernels_annihilate_constants_and_reproduce_linears(seed):
    rng = np.random.default_rng(seed)
    x = _random_tet(rng)
    c = np.array([1.3, -0.4, 2.0])
    # P1: A 1 = 0, and a(u_lin, v) = int grad u . grad v = |T| c . grad phi_i
    A1 = fo.p1_stiffness(x, ONE_CELL)[0]
    assert np.abs(A1.sum(axis=1)).max() < 1e-13 * np.abs(A1).max()
    # P2 with a P1 coefficient: A 1 = 0 for any k
    k = rng.uniform(0.5, 2.0, size=(1, 4))
    A2 = fo.p2_stiffness(x, ONE_CELL, k)[0]
    assert np.abs(A2.sum(axis=1)).max() < 1e-13 * np.abs(A2).max()
    assert np.allclose(A2, A2.T, atol=1e-14 * np.abs(A2).max())
    # P2 with constant k reproduces linear u exactly: A u_lin = k * int grad(u).grad(phi_i)
    A2c = fo.p2_stiffness(x, ONE_CELL, np.ones((1, 4)))[0]
    pts = [x[a] for a in range(4)] + [0.5 * (x[a] + x[b]) for a, b in fo.TET_EDGES]
    u = np.array([c @ p for p in pts])
    # int grad(phi_i) dx = boundary term; compare with P1 identity sum_j A_ij u_j = c . int grad phi_i
    J = (x[1:] - x[0]).T
    K = np.linalg.inv(J)
    adet = abs(np.linalg.det(J))
    R0 = fo.ref_grad_tensor(2, False)
    # int grad phi_i = |det| K^T int grad_hat phi_i ; int grad_hat phi_i = sum_j R0-like: use w and derivative
    gh = np.array([[fo._pint(fo._pdiff(p, a)) for a in range(3)] for p in fo._basis(2)], dtype=float)
    rhs = adet * gh @ K @ c
    assert np.allclose(A2c @ u, rhs, atol=1e-13 * np.abs(A2c).max())


@pytest.mark.parametrize("seed", [0, 1])
def test_elasticity_rigid_body_modes(seed):
    rng = np.random.default_rng(seed)
    x = _random_tet(rng)
    A = fo.p2_elasticity(x, ONE_CELL, np.array([1.7]), np.array([0.6]))[0]
    assert np.allclose(A, A.T, atol=1e-13 * np.abs(A).max())
    pts = np.array([x[a] for a in range(4)] + [0.5 * (x[a] + x[b]) for a, b in fo.TET_EDGES])
    modes = []
    for t in np.eye(3):
        modes.append(np.tile(t, 10))
    for w in np.eye(3):
        modes.append(np.cross(w, pts).reshape(-1))
    for r in modes:
        assert np.abs(A @ r).max() < 1e-12 * np.abs(A).max()


def test_nnz_closed_forms():
    for kind, n in [("p1", 3), ("p1", 5), ("p2", 2), ("p2", 4), ("vp2", 2)]:
        P = fo.build_problem(kind, n)
        rp, col = fo.sparsity(P["dofs"], P["dofs"], P["ndof"], P["bs"], P["bs"])
        assert len(col) == fo.nnz_formula(kind, n)
        # sorted unique columns per row, diagonal present
        for r in range(len(rp) - 1):
            seg = col[rp[r]:rp[r + 1]]
            assert np.all(np.diff(seg) > 0)
        assert np.all(fo.diag_positions(rp, col) >= 0)


def test_load_vector_integral_identities():
    # sum_i b_i = int f  (P2, DG0 f; P1 with P1 f)
    P = fo.build_problem("p2", 3)
    be = fo.element_vectors(P)
    _, det, _ = fo.cell_geometry(P["coords"], P["cells"])
    assert np.isclose(be.sum(), np.sum(np.abs(det) / 6 * P["f"]))
    P1 = fo.build_problem("p1", 3)
    b1 = fo.element_vectors(P1)
    _, det, _ = fo.cell_geometry(P1["coords"], P1["cells"])
    assert np.isclose(b1.sum(), np.sum(np.abs(det) / 6 * P1["f"][P1["cells"]].mean(axis=1)))


def test_patch_test_p2_dirichlet_solution_is_exact():
    # -div grad u = 0 with u = x + y + z on the boundary: P2 reproduces it exactly
    P = fo.build_problem("p2", 3)
    P["k"] = np.ones_like(P["k"])
    P["f"] = np.zeros_like(P["f"])
    S = fo.solve_system(P)
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    n = len(S["row_ptr"]) - 1
    A = sp.csr_matrix((S["A"], S["col"], S["row_ptr"]), shape=(n, n))
    u = spla.spsolve(A.tocsc(), S["b"])
    assert np.abs(u - P["g"]).max() < 1e-11


def test_pcg_matches_direct_solve():
    P = fo.build_problem("p2", 3)
    S = fo.solve_system(P)
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    n = len(S["row_ptr"]) - 1
    A = sp.csr_matrix((S["A"], S["col"], S["row_ptr"]), shape=(n, n))
    x_ref = spla.spsolve(A.tocsc(), S["b"])
    x, it = fo.pcg_jacobi(S["row_ptr"], S["col"], S["A"], S["b"], rtol=1e-12)
    assert it > 0 and np.abs(x - x_ref).max() < 1e-9 * np.abs(x_ref).max()


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_oracle_reproduces_golden_fixtures(path):
    G = np.load(path)
    kind = os.path.basename(path).split("_n")[0]
    P = fo.build_problem(kind, int(G["n"]), seed=0)
    S = fo.solve_system(P)
    assert np.array_equal(S["row_ptr"], G["row_ptr"]) and np.array_equal(S["col"], G["col"])
    assert np.array_equal(P["cells"], G["cells"]) and np.array_equal(P["dofs"], G["dofs"])
    scale = np.abs(G["A"]).max()
    assert np.abs(S["A"] - G["A"]).max() <= 1e-14 * scale
    assert np.abs(S["b"] - G["b"]).max() <= 1e-14 * max(1.0, np.abs(G["b"]).max())


@pytest.mark.parametrize("kind,n", [("p1", 5), ("p1k", 4), ("p2", 4), ("vp2", 3), ("p3", 3)])
def test_c_port_matches_numpy_oracle(kind, n):
    P = fo.build_problem(kind, n)
    S = fo.solve_system(P)
    C = cfem.CpuAssembler(P, S["row_ptr"], S["col"], nthreads=3)
    v = C.assemble_matrix().copy()
    b = C.assemble_rhs().copy()
    vb = C.matrix_bound()
    bb = C.rhs_bound()
    C.close()
    ok, worst = fo.within_bound(v, S["A"], S["A_bound"])
    assert ok, worst
    ok, worst = fo.within_bound(b, S["b"], S["b_bound"])
    assert ok, worst
    # the C port's bounds are the numpy oracle's (summed in another order)
    assert np.allclose(vb, S["A_bound"], rtol=1e-12, atol=0)
    assert np.allclose(bb, S["b_bound"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("kind,n", [("p1", 4), ("p2", 3), ("vp2", 2), ("p3", 2)])
def test_c_pattern_matches_numpy_oracle(kind, n):
    P = fo.build_problem(kind, n)
    rp, col = fo.sparsity(P["dofs"], P["dofs"], P["ndof"], P["bs"], P["bs"])
    for threads in (1, 3):
        rp_c, col_c = cfem.pattern(P["dofs"], P["ndof"], P["bs"], nthreads=threads)
        assert np.array_equal(rp_c, rp) and np.array_equal(col_c, col)


def test_exterior_facets_and_facet_tensors():
    for n in (1, 2, 3):
        coords, cells = fo.unit_cube_tet_mesh(n)
        F = fo.exterior_facets(cells)
        assert len(F) == 12 * n * n
        assert abs(fo.facet_areas(coords, cells, F).sum() - 6.0) < 1e-12
    coords, cells = fo.unit_cube_tet_mesh(3)
    F = fo.exterior_facets(cells)
    # sum of the facet mass = boundary area; P1 / P2 loads integrate g exactly
    for deg in (1, 2):
        M = fo.facet_mass(coords, cells, F, deg)
        assert abs(M.sum() - 6.0) < 1e-12
        assert np.allclose(M, np.transpose(M, (0, 2, 1)))
        assert abs(fo.facet_load(coords, cells, F, deg, 2.0).sum() - 12.0) < 1e-12
    # g = x + y + z as a P1 field: int_boundary g ds = 9 on the unit cube
    g = coords.sum(axis=1)
    for deg in (1, 2):
        b = fo.facet_load(coords, cells, F, deg, g, "p1", p1_cells=cells)
        assert abs(b.sum() - 9.0) < 1e-12
    t = fo.facet_vector_load(coords, cells, F, (1.0, -2.0, 0.5))
    assert np.allclose(t.reshape(len(F), 10, 3).sum(axis=(0, 1)), 6.0 * np.array([1.0, -2.0, 0.5]))


def test_exterior_facets_match_mirror_helper():
    from conftest import ensure_library  # noqa: F401
    from cudolfinx import fem
    for n in (2, 3):
        coords, cells = fo.unit_cube_tet_mesh(n)
        mesh = fem.create_unit_cube(n)
        assert np.array_equal(fem.exterior_facets(mesh), fo.exterior_facets(cells))


# --- equispaced P3 -----------------------------------------------------------
def _cube_gauss(fun, q=4):
    """Tensor Gauss-Legendre rule on [0,1]^3 (exact for degree 2q-1 per axis)."""
    t, w = np.polynomial.legendre.leggauss(q)
    t, w = 0.5 * (t + 1.0), 0.5 * w
    Z, Y, X = np.meshgrid(t, t, t, indexing="ij")
    W = (w[:, None, None] * w[None, :, None] * w[None, None, :]).ravel()
    return float(np.sum(W * fun(X.ravel(), Y.ravel(), Z.ravel())))


def _cubic(X):
    x, y, z = X[:, 0], X[:, 1], X[:, 2]
    return x ** 3 + y ** 2 * z + x * y * z - 2.0 * z ** 3


def _cubic_grad2(x, y, z):
    gx = 3 * x ** 2 + y * z
    gy = 2 * y * z + x * z
    gz = y ** 2 + x * y - 6 * z ** 2
    return gx * gx + gy * gy + gz * gz


def test_p3_basis_is_lagrange_and_integrals_known_answer():
    # phi_i(node_j) = delta_ij on the reference tet; int phi = |T|/40 (vertex),
    # 0 (edge), 9|T|/40 (face), |T| = 1/6
    B = fo._basis(3)
    W = fo.p3_local_points() / 3.0  # barycentric
    pts = W[:, 1:]  # reference coordinates (x, y, z) = (l1, l2, l3)
    V = np.array([[sum(float(c) * p[0] ** e[0] * p[1] ** e[1] * p[2] ** e[2] for e, c in phi.items())
                   for phi in B] for p in pts])
    assert np.abs(V - np.eye(20)).max() < 1e-14
    w3 = fo.ref_basis_integrals(3)
    assert np.allclose(w3[:4], 1.0 / 240) and np.allclose(w3[4:16], 0.0, atol=1e-17)
    assert np.allclose(w3[16:], 9.0 / 240)


@pytest.mark.parametrize("jitter", [0.0, 0.2])
def test_p3_energy_and_load_reproduce_cubic_integrals(jitter):
    # a cubic u is interpolated exactly: u^T A u = int |grad u|^2 and
    # sum_i b_i u_i = int u (f = 1) over the unit cube, on any affine mesh of it
    n = 3
    coords, cells = fo.unit_cube_tet_mesh(n, jitter=jitter, seed=4)
    dofs, ndof, _ = fo.p3_dofmap(n, cells)
    X = fo.dof_coordinates(coords, cells, dofs, ndof, 3)
    u = _cubic(X)
    Ae = fo.p3_stiffness(coords, cells)
    energy = np.einsum("ci,cij,cj->", u[dofs], Ae, u[dofs])
    assert abs(energy - _cube_gauss(_cubic_grad2)) < 1e-11 * energy
    be = fo.p3_load_dg0(coords, cells, np.ones(len(cells)))
    mean = np.einsum("ci,ci->", be, u[dofs])
    assert abs(mean - _cube_gauss(lambda x, y, z: x ** 3 + y ** 2 * z + x * y * z - 2 * z ** 3)) < 1e-13
    # constants are in the kernel of every element matrix
    assert np.abs(Ae.sum(axis=2)).max() < 1e-12 * np.abs(Ae).max()


def test_p3_patch_test_harmonic_cubic_is_exact():
    # -div grad u = 0 with a harmonic cubic on the boundary: P3 reproduces it
    P = fo.build_problem("p3", 2, seed=1)
    P["k"] = np.ones_like(P["k"])
    P["f"] = np.zeros_like(P["f"])
    X = fo.dof_coordinates(P["coords"], P["cells"], P["dofs"], P["ndof"], 3)
    P["g"] = X[:, 0] ** 3 - 3 * X[:, 0] * X[:, 1] ** 2 + X[:, 1] * X[:, 2]
    S = fo.solve_system(P)
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    m = len(S["row_ptr"]) - 1
    A = sp.csr_matrix((S["A"], S["col"], S["row_ptr"]), shape=(m, m))
    u = spla.spsolve(A.tocsc(), S["b"])
    assert np.abs(u - P["g"]).max() < 1e-11


def test_p3_nnz_closed_form_and_dof_count():
    for n in (1, 2, 3):
        P = fo.build_problem("p3", n)
        assert P["ndof"] == (3 * n + 1) ** 3
        rp, col = fo.sparsity(P["dofs"], P["dofs"], P["ndof"])
        assert len(col) == fo.nnz_formula("p3", n)
        assert np.diff(rp).max() <= 256  # block positions fit the byte map


# --- block / restricted systems ----------------------------------------------
def _csr(rp, col, vals, shape):
    import scipy.sparse as sp
    return sp.csr_matrix((vals, col, rp), shape=shape)


def _structural_submatrix(rp, col, rows, cols):
    """Pattern of A[rows][:, cols] (structural entries kept, explicit zeros too)."""
    import scipy.sparse as sp
    n = len(rp) - 1
    S = sp.csr_matrix((np.ones(len(col)), col, rp), shape=(n, n))[rows][:, cols].tocsr()
    S.sort_indices()
    return S.indptr.astype(np.int32), S.indices.astype(np.int32)


def test_block_system_block_diagonal_matches_separate_systems():
    import scipy.sparse as sp
    P1 = fo.build_problem("p1k", 3, seed=2)
    P2 = fo.build_problem("p2", 3, seed=2)
    S1, S2 = fo.solve_system(P1), fo.solve_system(P2)
    n1, n2 = P1["ndof"], P2["ndof"]
    parts = [(P1["dofs"], P1["dofs"], 1, 1, 0, 0), (P2["dofs"], P2["dofs"], 1, 1, n1, n1)]
    rp, col = fo.block_pattern(parts, n1 + n2, n1 + n2)
    blocks = []
    for P, off in ((P1, 0), (P2, n1)):
        mk = np.zeros(P["ndof"], dtype=np.uint8)
        mk[P["bc_dofs"]] = 1
        blocks.append(dict(Ae=fo.element_matrices(P), dofs0=P["dofs"], dofs1=P["dofs"], bs0=1, bs1=1, row_offset=off,
                           col_offset=off, markers0=mk, markers1=mk, bc_rows=P["bc_dofs"]))
    v = fo.assemble_block_matrix(blocks, rp, col)
    ref = sp.block_diag([_csr(S1["row_ptr"], S1["col"], S1["A"], (n1, n1)),
                         _csr(S2["row_ptr"], S2["col"], S2["A"], (n2, n2))]).tocsr()
    ref.sort_indices()
    assert np.array_equal(rp, ref.indptr) and np.array_equal(col, ref.indices)
    assert np.array_equal(v, ref.data)


@pytest.mark.parametrize("kind,bs", [("p2", 1), ("vp2", 3)])
def test_restricted_system_is_the_submatrix_of_the_full_system(kind, bs):
    # dofs outside a restriction take no entries: the restricted matrix is
    # A_full[R, R] (pattern and values), for any restriction
    P = fo.build_problem(kind, 3, seed=5)
    dofs, nd = P["dofs"], P["ndof"]
    X = fo.dof_coordinates(P["coords"], P["cells"], dofs, nd, 2)
    R = np.nonzero(X[:, 0] <= 0.5 + 1e-12)[0]
    Ae = fo.element_matrices(P)
    rp_f, col_f = fo.sparsity(dofs, dofs, nd, bs, bs)
    A_f = fo.assemble_matrix(Ae, dofs, dofs, rp_f, col_f, bs, bs)
    dr = fo.restricted_dofmap(dofs, R, nd)
    nr = len(R) * bs
    rp, col = fo.block_pattern([(dr, dr, bs, bs, 0, 0)], nr, nr)
    v = fo.assemble_block_matrix([dict(Ae=Ae, dofs0=dr, dofs1=dr, bs0=bs, bs1=bs, row_offset=0, col_offset=0)],
                                 rp, col)
    keep = (R[:, None] * bs + np.arange(bs)).ravel()
    srp, scol = _structural_submatrix(rp_f, col_f, keep, keep)
    assert np.array_equal(rp, srp) and np.array_equal(col, scol)
    sub = _csr(rp_f, col_f, A_f, (nd * bs, nd * bs))[keep][:, keep].tocsr()
    sub.sort_indices()
    assert np.allclose(v, sub.data, rtol=0, atol=1e-14 * np.abs(A_f).max())
    # restricted load vector = the kept entries of the full one
    if kind == "p2":
        be = fo.element_vectors(P)
        b_full = fo.assemble_vector(be, dofs, nd)
        b = fo.assemble_block_vector([(be, dr, 1, 0)], len(R))
        assert np.allclose(b, b_full[R], rtol=0, atol=1e-15)


def test_coupled_restricted_block_system_is_a_submatrix():
    # [[K, -K], [-K, 2K]] on (V, V_R): the second field restricted to x <= 1/2;
    # equals the unrestricted 2x2 system with the excluded rows / columns of
    # the second field removed, BC rows included
    import scipy.sparse as sp
    P = fo.build_problem("p2", 3, seed=9)
    dofs, nd = P["dofs"], P["ndof"]
    X = fo.dof_coordinates(P["coords"], P["cells"], dofs, nd, 2)
    R = np.nonzero(X[:, 0] <= 0.5 + 1e-12)[0]
    K = fo.element_matrices(P)
    mk = np.zeros(nd, dtype=np.uint8)
    mk[P["bc_dofs"]] = 1

    def system(d1, n1, mk1, bc1):
        parts = [(dofs, dofs, 1, 1, 0, 0), (dofs, d1, 1, 1, 0, nd), (d1, dofs, 1, 1, nd, 0), (d1, d1, 1, 1, nd, nd)]
        rp, col = fo.block_pattern(parts, nd + n1, nd + n1)
        B = [dict(Ae=K, dofs0=dofs, dofs1=dofs, row_offset=0, col_offset=0, markers0=mk, markers1=mk,
                  bc_rows=P["bc_dofs"]),
             dict(Ae=-K, dofs0=dofs, dofs1=d1, row_offset=0, col_offset=nd, markers0=mk, markers1=mk1,
                  bc_rows=P["bc_dofs"]),
             dict(Ae=-K, dofs0=d1, dofs1=dofs, row_offset=nd, col_offset=0, markers0=mk1, markers1=mk, bc_rows=bc1),
             dict(Ae=2 * K, dofs0=d1, dofs1=d1, row_offset=nd, col_offset=nd, markers0=mk1, markers1=mk1,
                  bc_rows=bc1)]
        for b in B:
            b.update(bs0=1, bs1=1)
        return rp, col, fo.assemble_block_matrix(B, rp, col)

    rp_f, col_f, v_f = system(dofs, nd, mk, P["bc_dofs"])
    dr = fo.restricted_dofmap(dofs, R, nd)
    mkr = mk[R]
    rp, col, v = system(dr, len(R), mkr, np.nonzero(mkr)[0])
    keep = np.concatenate([np.arange(nd), nd + R])
    srp, scol = _structural_submatrix(rp_f, col_f, keep, keep)
    assert np.array_equal(rp, srp) and np.array_equal(col, scol)
    sub = _csr(rp_f, col_f, v_f, (2 * nd, 2 * nd))[keep][:, keep].tocsr()
    sub.sort_indices()
    assert np.allclose(v, sub.data, rtol=0, atol=1e-14 * np.abs(v_f).max())


# --- interpolation ------------------------------------------------------------
@pytest.mark.parametrize("dt,ds", [(1, 1), (2, 1), (3, 1), (3, 2), (1, 2), (2, 3), (0, 1), (0, 2)])
def test_interpolation_operator_reproduces_the_source_polynomials(dt, ds):
    # IM maps the source nodal values of any polynomial of the source degree to
    # its values at the target nodes
    rng = np.random.default_rng(dt * 7 + ds)
    c = rng.standard_normal(10)

    def poly(X):  # a quadratic (exact in P2 / P3, its linear part in P1)
        x, y, z = X[:, 0], X[:, 1], X[:, 2]
        q = c[0] + c[1] * x + c[2] * y + c[3] * z
        if ds >= 2:
            q = q + c[4] * x * x + c[5] * x * y + c[6] * y * z + c[7] * z * z + c[8] * x * z + c[9] * y * y
        return q

    im = fo.interpolation_operator(dt, ds)
    got = im @ poly(fo.element_nodes(ds))
    assert np.allclose(got, poly(fo.element_nodes(dt)), atol=1e-13)


def test_oracle_interpolation_is_exact_for_polynomials_on_the_mesh():
    n = 3
    coords, cells = fo.unit_cube_tet_mesh(n, jitter=0.2, seed=3)
    d2, n2, _ = fo.p2_dofmap(n, cells)
    d3, n3, _ = fo.p3_dofmap(n, cells)
    X2 = fo.dof_coordinates(coords, cells, d2, n2, 2)
    X3 = fo.dof_coordinates(coords, cells, d3, n3, 3)
    q = lambda X: 1 + X[:, 0] - 2 * X[:, 1] * X[:, 2] + X[:, 2] ** 2
    u3 = fo.interpolate_same_map(q(X2), d2, d3, fo.interpolation_operator(3, 2), n3)
    assert np.abs(u3 - q(X3)).max() < 1e-13
    u2 = fo.interpolate_same_map(u3, d3, d2, fo.interpolation_operator(2, 3), n2)
    assert np.abs(u2 - q(X2)).max() < 1e-13


# --- interior-facet (DG) integrals ----------------------------------------------
def _dg_problem(n=3, jitter=0.2, seed=1):
    coords, cells = fo.unit_cube_tet_mesh(n, jitter=jitter, seed=seed)
    return coords, cells, fo.interior_facets(cells)


def test_interior_facets_pair_matching_faces():
    coords, cells, q = _dg_problem(3)
    n = 3
    # every facet is interior or exterior; 4 facets per cell
    ext = fo.exterior_facets(cells)
    assert 2 * len(q) + len(ext) == 4 * len(cells)
    assert len(ext) == 2 * 6 * n * n  # two triangles per boundary square
    F = np.array(fo.TET_FACETS)
    a = np.sort(cells[q[:, 0][:, None], F[q[:, 1]]], axis=1)
    b = np.sort(cells[q[:, 2][:, None], F[q[:, 3]]], axis=1)
    assert np.array_equal(a, b) and np.all(q[:, 0] < q[:, 2])


def test_dg0_jump_matrix_is_the_area_weighted_cell_graph_laplacian():
    coords, cells, q = _dg_problem(2)
    C = len(cells)
    alpha = np.random.default_rng(0).uniform(0.5, 2.0, C)
    af = fo.facet_average(alpha, q)
    Ae = fo.interior_jump_tensors(coords, cells, q, 0, af)
    d = fo.dg_dofmap(C, 0)
    A = np.zeros((C, C))
    for f, (c0, _, c1, _) in enumerate(q):
        m = fo.macro_dofmap(d, q[f:f + 1])[0]
        A[np.ix_(m, m)] += Ae[f]
    area = fo.facet_areas(coords, cells, q[:, :2])
    L = np.zeros((C, C))
    for f, (c0, _, c1, _) in enumerate(q):
        w = af[f] * area[f]
        L[c0, c0] += w
        L[c1, c1] += w
        L[c0, c1] -= w
        L[c1, c0] -= w
    assert np.allclose(A, L, rtol=1e-13, atol=1e-15)


def test_dg1_jump_vanishes_on_continuous_fields_and_is_the_jump_norm():
    coords, cells, q = _dg_problem(3)
    C = len(cells)
    d = fo.dg_dofmap(C, 1)
    m = fo.macro_dofmap(d, q)
    Ae = fo.interior_jump_tensors(coords, cells, q, 1)
    rng = np.random.default_rng(4)
    # a continuous P1 field written into DG1 has no jump
    uc = rng.standard_normal(len(coords))[cells].ravel()
    assert np.abs(np.einsum("fij,fj->fi", Ae, uc[m])).max() < 1e-14
    assert abs(fo.interior_jump_norm(coords, cells, q, 1, uc[m])) < 1e-28
    # for any DG1 field, u^T A u is the jump norm
    u = rng.standard_normal(4 * C)
    uAu = np.einsum("fi,fij,fj->", u[m], Ae, u[m])
    assert abs(uAu - fo.interior_jump_norm(coords, cells, q, 1, u[m])) < 1e-12 * uAu


def test_interior_average_load_sums_to_the_interior_facet_area():
    coords, cells, q = _dg_problem(3)
    area = fo.facet_areas(coords, cells, q[:, :2]).sum()
    for degree in (0, 1):
        be = fo.interior_avg_load(coords, cells, q, degree)
        assert abs(be.sum() - area) < 1e-13 * area


@pytest.mark.parametrize("kind", ["p1k", "p2", "p3", "vp2"])
def test_diagonal_part_is_the_diagonal_of_the_matrix_without_bcs(kind):
    P = fo.build_problem(kind, 2, seed=3)
    bs, dofs = P["bs"], P["dofs"]
    rp, col = fo.sparsity(dofs, dofs, P["ndof"], bs, bs)
    Ae = fo.element_matrices(P)
    A = fo.assemble_matrix(Ae, dofs, dofs, rp, col, bs, bs)
    d = fo.assemble_diagonal(Ae, dofs, P["ndof"] * bs, bs)
    assert np.allclose(d, A[fo.diag_positions(rp, col)], rtol=1e-14, atol=0)
    assert np.all(d > 0)  # an SPD operator's diagonal


def _collapsed_gauss(q=6):
    """Points/weights on the reference tet from a tensor Gauss rule on the cube
    (x = u, y = v (1-u), z = w (1-u)(1-v)), exact for polynomials of degree
    <= 2q - 3 -- independent of the exact monomial integration."""
    t, w = np.polynomial.legendre.leggauss(q)
    t, w = 0.5 * (t + 1.0), 0.5 * w
    U, V, W = np.meshgrid(t, t, t, indexing="ij")
    WU, WV, WW = np.meshgrid(w, w, w, indexing="ij")
    x = U
    y = V * (1 - U)
    z = W * (1 - U) * (1 - V)
    wt = WU * WV * WW * (1 - U) ** 2 * (1 - V)
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1), wt.ravel()


def _eval_poly(p, X):
    return sum(float(v) * X[:, 0] ** k[0] * X[:, 1] ** k[1] * X[:, 2] ** k[2] for k, v in p.items())


@pytest.mark.parametrize("degree", [1, 2])
def test_mass_tensors_match_an_independent_quadrature(degree):
    X, w = _collapsed_gauss()
    phi = np.array([_eval_poly(p, X) for p in fo._basis(degree)])
    lam = np.array([_eval_poly(p, X) for p in fo._LAMBDA])
    M0 = np.einsum("iq,jq,q->ij", phi, phi, w)
    M = np.einsum("mq,iq,jq,q->mij", lam, phi, phi, w)
    assert np.allclose(fo.ref_mass_tensor(degree, False), M0, rtol=0, atol=1e-15)
    assert np.allclose(fo.ref_mass_tensor(degree, True), M, rtol=0, atol=1e-15)
    assert abs(fo.ref_mass_tensor(degree, False).sum() - 1.0 / 6.0) < 1e-15  # partition of unity
    if degree == 1:
        expect = (np.ones((4, 4)) + np.eye(4)) / 120.0  # int lambda_i lambda_j = (1 + delta_ij) |T| / 20
        assert np.allclose(fo.ref_mass_tensor(1, False), expect, rtol=0, atol=1e-17)


def test_mass_matrix_reproduces_l2_norms_of_polynomials():
    # u in the space: u^T M u = int u^2 over the unit cube, on a jittered mesh
    coords, cells = fo.unit_cube_tet_mesh(3, jitter=0.2, seed=4)
    x, y, z = coords[:, 0], coords[:, 1], coords[:, 2]
    u = 1.0 + x - 2.0 * y + 3.0 * z
    Ae = fo.mass_matrices(coords, cells, 1)
    rp, col = fo.sparsity(cells, cells, len(coords))
    M = fo.assemble_matrix(Ae, cells, cells, rp, col)
    import scipy.sparse as sp
    Ms = sp.csr_matrix((M, col, rp), shape=(len(coords), len(coords)))
    # int_[0,1]^3 (1 + x - 2y + 3z)^2 = 1 + (1+4+9)/3 + 2*(1-2+3)/2 + 2*(-2+3-6)/4 = 6.4166...
    exact = 1 + 14 / 3 + 2 + 2 * (1 * -2 + 1 * 3 + -2 * 3) / 4
    assert abs(u @ (Ms @ u) - exact) < 1e-12 * exact


def test_vector_mass_reproduces_the_l2_norm_of_a_quadratic_vector_field():
    import scipy.sparse as sp
    n = 3
    coords, cells = fo.unit_cube_tet_mesh(n, jitter=0.2, seed=9)
    dofs, ndof, _ = fo.p2_dofmap(n, cells)
    X = fo.dof_coordinates(coords, cells, dofs, ndof, 2)
    x, y, z = X[:, 0], X[:, 1], X[:, 2]
    u = np.stack([x * x, y * z, np.ones_like(x)], axis=1).ravel()
    Ae = fo.vector_mass(fo.mass_matrices(coords, cells, 2, c_dg0=np.full(len(cells), 2.0)))
    rp, col = fo.sparsity(dofs, dofs, ndof, 3, 3)
    M = sp.csr_matrix((fo.assemble_matrix(Ae, dofs, dofs, rp, col, 3, 3), col, rp), shape=(3 * ndof, 3 * ndof))
    exact = 2.0 * (1 / 5 + 1 / 9 + 1.0)
    assert abs(u @ (M @ u) - exact) < 1e-12 * exact
