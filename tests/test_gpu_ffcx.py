"""Forms given as FFCx tabulate_tensor bodies (fe_form_create_ffcx), on the GPU
against the oracle.

The reference assembles any UFL form by wrapping the tabulate_tensor bodies
FFCx generates (python/cudolfinx/jit.py:15-114) into NVRTC-compiled kernels
(cpp/cudolfinx/fem/CUDAFormIntegral.cpp:2366-2558); its tests assemble
nonlinear residuals, Jacobians and functionals over cells, exterior and
interior facets (python/test/test_cuda_assembly.py:48-91).  The bodies here
are hand-written in FFCx's format (tests/ffcx_bodies.py); the engine compiles
them with NVRTC inside its own skeletons.  Bars: patterns bit-exact with the
oracle's; values within the oracle's per-entry bound (fem_oracle.matrix_bound
/ vector_bound / lifting_bound), against the exact element tensors where the
integrand is polynomial (stiffness, mass, elasticity, mixed P2-P1, Robin,
jump penalty) and against the oracle's numpy evaluation of the same
quadrature elsewhere (exp(u) forms, facet normals, SIPG).  Interior-facet
bodies read per-side permuted tables, the oracle locates the points on the
second cell by its own barycentric solve, so a wrong permutation shows.
"""
import numpy as np
import pytest

import ffcx_bodies as fb
from conftest import ensure_library
from gpu_util import tolerance_check
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


def _cx():
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem
    return cx, fem


def _integral(B, entities=None):
    from cudolfinx import fem
    return fem.FFCxIntegral(B["integral_type"], B["name"], B["body"], entities)


def _mesh(n=3, jitter=0.2, seed=1, relabel=False):
    """Jittered unit cube; `relabel` renumbers the vertices at random so that
    interior facets take all six quadrature permutations."""
    cx, fem = _cx()
    coords, cells = fo.unit_cube_tet_mesh(n, jitter=jitter, seed=seed)
    if relabel:
        perm = np.random.default_rng(seed).permutation(len(coords))
        coords = coords[np.argsort(perm)]
        cells = perm[cells].astype(np.int32)
    return cx, fem, fem.Mesh(coords, cells, grid_n=None if relabel else n), coords, cells


def _bcs_p1(fem, V, coords, g=None):
    grid = np.nonzero((np.abs(coords) < 1e-12).any(axis=1) | (np.abs(coords - 1) < 1e-12).any(axis=1))[0]
    gv = np.zeros(V.num_dofs) if g is None else g
    return fem.dirichletbc(fem.Function(V, gv), grid.astype(np.int32)), grid


def _markers(n, dofs):
    m = np.zeros(n, dtype=np.uint8)
    m[dofs] = 1
    return m


@pytest.mark.parametrize("k_kind", ["dg0", "p1"])
def test_stiffness_bodies_match_the_oracle_and_the_builtin_kernels(k_kind):
    cx, fem, mesh, coords, cells = _mesh(3, jitter=0.0)
    for degree in (1, 2):
        V = fem.functionspace(mesh, ("P", degree))
        rng = np.random.default_rng(degree)
        if k_kind == "dg0":
            kv = np.exp(rng.standard_normal(mesh.num_cells))
            k = fem.Function(fem.functionspace(mesh, ("DG", 0)), kv)
            kc = kv
        else:
            kv = np.exp(rng.standard_normal(mesh.num_vertices))
            k = fem.Function(fem.functionspace(mesh, ("P", 1)), kv)
            kc = kv[cells]
        if degree == 1 and k_kind == "p1":
            continue  # the built-in P1 kernel takes the exact cell mean; covered by P2 here
        B = fb.stiffness(degree, k_kind)
        a = cx.form(fem.FFCxForm([_integral(B)], [V, V], [k]))
        bc, bdofs = _bcs_p1(fem, V, V.tabulate_dof_coordinates(), V.tabulate_dof_coordinates().sum(axis=1))
        asm = cx.CUDAAssembler()
        A = asm.assemble_matrix(a, bcs=[bc])
        A.assemble()
        rp, col = A.sparsity.to_host()
        rp_o, col_o = fo.sparsity(V.dofs, V.dofs, V.num_nodes)
        assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o)
        mk = _markers(V.num_dofs, bdofs)
        if degree == 1:
            Ae = fo.p1_stiffness(coords, cells, kv)
        else:
            Ae = fo.p2_stiffness(coords, cells, kc if k_kind == "p1" else np.repeat(kc[:, None], 4, axis=1))
        ref = fo.assemble_matrix(Ae, V.dofs, V.dofs, rp_o, col_o, 1, 1, mk, mk, 1.0, bdofs)
        bound = fo.matrix_bound(Ae, V.dofs, V.dofs, rp_o, col_o, 1, 1, mk, mk)
        ok, worst = tolerance_check(A.values.cpu().numpy(), ref, bound)
        assert ok, (degree, worst)
        # the built-in kernel on the same inputs lies within the same bound
        A2 = asm.assemble_matrix(cx.form(fem.stiffness(V, k)), bcs=[bc])
        A2.assemble()
        ok, worst = tolerance_check(A2.values.cpu().numpy(), ref, bound)
        assert ok, (degree, worst)
        # lifting through the body, then set_bc
        L = cx.form(fem.load(V, 0.0))
        b = asm.assemble_vector(L)
        asm.apply_lifting(b, [a], [[bc]])
        g = bc.value.x.array
        ref_b = fo.apply_lifting(np.zeros(V.num_dofs), Ae, V.dofs, V.dofs, mk, g)
        ok, worst = tolerance_check(b.to_host(), ref_b, fo.lifting_bound(V.num_dofs, Ae, V.dofs, V.dofs, mk, g))
        assert ok, (degree, worst)


def test_a_form_without_a_builtin_kind_with_a_constant():
    # k * grad u . grad v + c * u * v: stiffness with a DG0 k plus a mass term
    # scaled by a Constant; the constant is re-read on every assembly
    cx, fem, mesh, coords, cells = _mesh(3)
    V = fem.functionspace(mesh, ("P", 1))
    kv = np.random.default_rng(3).uniform(0.5, 2.0, mesh.num_cells)
    k = fem.Function(fem.functionspace(mesh, ("DG", 0)), kv)
    spec = fem.FFCxForm([_integral(fb.stiffness_plus_mass())], [V, V], [k], [2.5])
    a = cx.form(spec)
    asm = cx.CUDAAssembler()
    rp, col = fo.sparsity(V.dofs, V.dofs, V.num_nodes)
    K = fo.p1_stiffness(coords, cells, kv)
    M = fo.mass_matrices(coords, cells, 1)
    for c in (2.5, -0.75):
        spec.constants[0] = c
        A = asm.assemble_matrix(a)
        A.assemble()
        ref = fo.assemble_matrix(K + c * M, V.dofs, V.dofs, rp, col)
        bound = fo.matrix_bound(K, V.dofs, V.dofs, rp, col) + fo.matrix_bound(c * M, V.dofs, V.dofs, rp, col)
        ok, worst = tolerance_check(A.values.cpu().numpy(), ref, bound)
        assert ok, (c, worst)


def test_blocked_vector_p2_elasticity_body():
    cx, fem, mesh, coords, cells = _mesh(2)
    V = fem.functionspace(mesh, ("P", 2, (3,)))
    W = fem.functionspace(mesh, ("DG", 0))
    rng = np.random.default_rng(4)
    lam, mu = rng.uniform(0.5, 2.0, mesh.num_cells), rng.uniform(0.2, 1.0, mesh.num_cells)
    a = cx.form(fem.FFCxForm([_integral(fb.elasticity())], [V, V], [fem.Function(W, lam), fem.Function(W, mu)]))
    A = cx.CUDAAssembler().assemble_matrix(a)
    A.assemble()
    rp, col = A.sparsity.to_host()
    Ae = fo.p2_elasticity(coords, cells, lam, mu)
    ref = fo.assemble_matrix(Ae, V.dofs, V.dofs, rp, col, 3, 3)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref, fo.matrix_bound(Ae, V.dofs, V.dofs, rp, col, 3, 3))
    assert ok, worst


def test_mixed_element_p2_p1_coupling_block():
    # int p dv/dx dx, v in P2, p in P1: a rectangular block of a mixed system
    cx, fem, mesh, coords, cells = _mesh(3)
    V = fem.functionspace(mesh, ("P", 2))
    Q = fem.functionspace(mesh, ("P", 1))
    a = cx.form(fem.FFCxForm([_integral(fb.mixed_p2_p1())], [V, Q]))
    A = cx.CUDAAssembler().assemble_matrix(a)
    A.assemble()
    rp, col = A.sparsity.to_host()
    rp_o, col_o = fo.sparsity(V.dofs, Q.dofs, V.num_nodes)
    assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o)
    Ae = fo.quad_cell_matrix(coords, cells, 2, 1, lambda V0, G0, V1, G1: G0[..., :, None, 0] * V1[None, :, None, :],
                             n=3)
    ref = fo.assemble_matrix(Ae, V.dofs, Q.dofs, rp_o, col_o)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref, fo.matrix_bound(Ae, V.dofs, Q.dofs, rp_o, col_o))
    assert ok, worst


def test_nonlinear_cell_residual_jacobian_and_functional():
    # (exp(u) kappa v + grad u . grad v) dx, its derivative and exp(u) kappa dx
    cx, fem, mesh, coords, cells = _mesh(3)
    V = fem.functionspace(mesh, ("P", 1))
    X = coords
    uv = X[:, 0] ** 2 + X[:, 1]
    kv = np.sin(X[:, 0]) * np.cos(X[:, 1])
    u, kappa = fem.Function(V, uv), fem.Function(V, kv)
    asm = cx.CUDAAssembler()
    R, Jm, Mv = fo.quad_cell_forms(coords, cells, uv[cells], kv[cells], n=4)
    F = cx.form(fem.FFCxForm([_integral(fb.nonlinear(1))], [V], [u, kappa]))
    b = asm.assemble_vector(F).to_host()
    ok, worst = tolerance_check(b, fo.assemble_vector(R, V.dofs, V.num_dofs), fo.vector_bound(R, V.dofs, V.num_dofs))
    assert ok, worst
    Jf = cx.form(fem.FFCxForm([_integral(fb.nonlinear(2))], [V, V], [u, kappa]))
    bc, bdofs = _bcs_p1(fem, V, X, X.sum(axis=1))
    A = asm.assemble_matrix(Jf, bcs=[bc])
    A.assemble()
    rp, col = A.sparsity.to_host()
    mk = _markers(V.num_dofs, bdofs)
    ref = fo.assemble_matrix(Jm, V.dofs, V.dofs, rp, col, 1, 1, mk, mk, 1.0, bdofs)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref, fo.matrix_bound(Jm, V.dofs, V.dofs, rp, col, 1, 1, mk, mk))
    assert ok, worst
    val = asm.assemble_scalar(cx.form(fem.FFCxForm([_integral(fb.nonlinear(0))], [], [u, kappa])))
    ref_val = float(np.sum(Mv))
    assert abs(val - ref_val) <= 1e-12 * np.abs(Mv).sum()
    # a coefficient update reaches the next assembly
    u.x.array[:] = 0.5 * uv
    R2, _, _ = fo.quad_cell_forms(coords, cells, 0.5 * uv[cells], kv[cells], n=4)
    b2 = asm.assemble_vector(F).to_host()
    ok, worst = tolerance_check(b2, fo.assemble_vector(R2, V.dofs, V.num_dofs), fo.vector_bound(R2, V.dofs, V.num_dofs))
    assert ok, worst


def test_exterior_facet_bodies_and_a_two_integral_form():
    cx, fem, mesh, coords, cells = _mesh(3)
    V = fem.functionspace(mesh, ("P", 1))
    F = fo.exterior_facets(cells)
    asm = cx.CUDAAssembler()
    rng = np.random.default_rng(6)
    alpha = rng.uniform(0.5, 2.0, mesh.num_cells)
    W = fem.functionspace(mesh, ("DG", 0))
    # Robin mass alone, and dx stiffness + ds Robin as one form of two integrals
    rob = fem.FFCxForm([_integral(fb.robin_mass(1))], [V, V], [fem.Function(W, alpha)])
    A = asm.assemble_matrix(cx.form(rob))
    A.assemble()
    rp, col = A.sparsity.to_host()
    Ae = fo.facet_mass(coords, cells, F, 1, alpha[F[:, 0]])
    fd = V.dofs[F[:, 0]]
    ref = fo.assemble_matrix(Ae, fd, fd, rp, col)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref, fo.matrix_bound(Ae, fd, fd, rp, col))
    assert ok, worst
    two = fem.FFCxForm([_integral(fb.stiffness(1, "dg0")), _integral(fb.robin_mass(1))], [V, V],
                       [fem.Function(W, alpha)])
    A2 = asm.assemble_matrix(cx.form(two))
    A2.assemble()
    K = fo.p1_stiffness(coords, cells, alpha)
    ref2 = ref + fo.assemble_matrix(K, V.dofs, V.dofs, rp, col)
    bound2 = fo.matrix_bound(Ae, fd, fd, rp, col) + fo.matrix_bound(K, V.dofs, V.dofs, rp, col)
    ok, worst = tolerance_check(A2.values.cpu().numpy(), ref2, bound2)
    assert ok, worst
    # u kappa v (grad u . n) ds and its derivative (the reference's exterior forms)
    uv = coords[:, 0] ** 2 + coords[:, 1]
    kv = np.sin(coords[:, 0]) * np.cos(coords[:, 1])
    u, kappa = fem.Function(V, uv), fem.Function(V, kv)
    Rf, Jf = fo.exterior_facet_forms(coords, cells, F, uv[cells], kv[cells], n=3)
    b = asm.assemble_vector(cx.form(fem.FFCxForm([_integral(fb.exterior_nonlinear(1), F)], [V], [u, kappa])))
    ok, worst = tolerance_check(b.to_host(), fo.assemble_vector(Rf, fd, V.num_dofs), fo.vector_bound(Rf, fd, V.num_dofs))
    assert ok, worst
    A3 = asm.assemble_matrix(cx.form(fem.FFCxForm([_integral(fb.exterior_nonlinear(2), F)], [V, V], [u, kappa])))
    A3.assemble()
    ok, worst = tolerance_check(A3.values.cpu().numpy(), fo.assemble_matrix(Jf, fd, fd, rp, col),
                                fo.matrix_bound(Jf, fd, fd, rp, col))
    assert ok, worst


def test_interior_facet_bodies_with_permuted_tables():
    cx, fem, mesh, coords, cells = _mesh(3, relabel=True)
    q = fo.interior_facets(cells)
    codes = {fo.facet_permutation(cells[c][list(fo.TET_FACETS[f])]) for c, f in zip(q[:, 0], q[:, 1])}
    assert codes == set(range(6))  # every permutation occurs
    V = fem.functionspace(mesh, ("DG", 1))
    P1 = fem.functionspace(mesh, ("P", 1))
    asm = cx.CUDAAssembler()
    d = fo.dg_dofmap(mesh.num_cells, 1)
    m = fo.macro_dofmap(d, q)
    N = V.num_dofs
    # jump penalty: the same matrix as the exact oracle and the built-in DG1 kernel
    a = cx.form(fem.FFCxForm([_integral(fb.interior_jump())], [V, V], [], [3.0]))
    A = asm.assemble_matrix(a)
    A.assemble()
    rp, col = A.sparsity.to_host()
    rp_o, col_o = fo.sparsity(m, m, N)
    assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o)
    Aj = fo.interior_jump_tensors(coords, cells, q, 1, np.full(len(q), 3.0))
    ok, worst = tolerance_check(A.values.cpu().numpy(), fo.assemble_matrix(Aj, m, m, rp_o, col_o),
                                fo.matrix_bound(Aj, m, m, rp_o, col_o))
    assert ok, worst
    # a continuous field has no jumps: u^T A u = sum of int jump(u)^2 = 0 only
    # when both sides' tables sample the same physical points
    import scipy.sparse as sp
    Aj_csr = sp.csr_matrix((A.values.cpu().numpy(), col, rp), shape=(N, N))
    up = (coords[:, 0] - 2.0 * coords[:, 1] + 0.5 * coords[:, 2])[cells].ravel()  # P1 values copied into DG1
    ref_scale = np.abs(up) @ (abs(Aj_csr) @ np.abs(up))
    assert abs(up @ (Aj_csr @ up)) <= 1e-12 * ref_scale
    # SIPG with normal derivatives
    R, Jm, Mv, S = fo.interior_facet_forms(coords, cells, q, np.zeros((mesh.num_cells, 4)),
                                           np.zeros(mesh.num_vertices), cells, 7.0, n=3)
    A = asm.assemble_matrix(cx.form(fem.FFCxForm([_integral(fb.interior_sipg())], [V, V], [], [7.0])))
    A.assemble()
    ok, worst = tolerance_check(A.values.cpu().numpy(), fo.assemble_matrix(S, m, m, rp_o, col_o),
                                fo.matrix_bound(S, m, m, rp_o, col_o))
    assert ok, worst
    # nonlinear residual, Jacobian and functional with DG1 u and P1 kappa
    X = coords
    uv = np.random.default_rng(8).standard_normal((mesh.num_cells, 4))
    kv = np.sin(X[:, 0]) * np.cos(X[:, 1])
    u, kappa = fem.Function(V, uv.ravel()), fem.Function(P1, kv)
    R, Jm, Mv, _ = fo.interior_facet_forms(coords, cells, q, uv, kv, cells, 0.0, n=3)
    b = asm.assemble_vector(cx.form(fem.FFCxForm([_integral(fb.interior_nonlinear(1))], [V], [u, kappa])))
    ok, worst = tolerance_check(b.to_host(), fo.assemble_vector(R, m, N), fo.vector_bound(R, m, N))
    assert ok, worst
    A = asm.assemble_matrix(cx.form(fem.FFCxForm([_integral(fb.interior_nonlinear(2))], [V, V], [u, kappa])))
    A.assemble()
    ok, worst = tolerance_check(A.values.cpu().numpy(), fo.assemble_matrix(Jm, m, m, rp_o, col_o),
                                fo.matrix_bound(Jm, m, m, rp_o, col_o))
    assert ok, worst
    val = asm.assemble_scalar(cx.form(fem.FFCxForm([_integral(fb.interior_nonlinear(0))], [], [u, kappa],
                                                   domain=mesh)))
    assert abs(val - Mv.sum()) <= 1e-12 * np.abs(Mv).sum()


def test_compile_errors_cache_and_argument_checks(tmp_path):
    cx, fem, mesh, coords, cells = _mesh(2)
    V = fem.functionspace(mesh, ("P", 1))
    bad = fem.FFCxIntegral("cell", "tabulate_tensor_integral_bad", "  A[0] += undefined_symbol;\n")
    with pytest.raises(RuntimeError, match="NVRTC"):
        cx.form(fem.FFCxForm([bad], [V, V]))
    B = fb.stiffness(1, "dg0")
    W = fem.functionspace(mesh, ("DG", 0))
    k = fem.Function(W, np.ones(mesh.num_cells))
    # the coefficient's element must have the declared number of values per cell
    with pytest.raises(RuntimeError, match="values per cell"):
        cx.form(fem.FFCxForm([_integral(B)], [V, V], [fem.Function(V, np.ones(V.num_dofs))],
                             coefficient_sizes=B["coefficient_sizes"]))
    # on-disk cache: the second form loads the cubin written by the first
    a1 = cx.form(fem.FFCxForm([_integral(B)], [V, V], [k]), cachedir=str(tmp_path))
    files = sorted(p.name for p in tmp_path.iterdir())
    assert any(f.endswith(".cubin") for f in files) and any(f.endswith(".cu") for f in files)
    a2 = cx.form(fem.FFCxForm([_integral(B)], [V, V], [k]), cachedir=str(tmp_path))
    asm = cx.CUDAAssembler()
    A1 = asm.assemble_matrix(a1)
    A2 = asm.assemble_matrix(a2)
    A1.assemble()
    A2.assemble()
    rp, col = A1.sparsity.to_host()
    Ae = fo.p1_stiffness(coords, cells)
    for A in (A1, A2):
        ok, worst = tolerance_check(A.values.cpu().numpy(), fo.assemble_matrix(Ae, V.dofs, V.dofs, rp, col),
                                    fo.matrix_bound(Ae, V.dofs, V.dofs, rp, col))
        assert ok, worst
    # FFCx forms assemble with the atomic scatter only
    with pytest.raises(RuntimeError, match="atomic scatter only"):
        asm.assemble_matrix(a1, variant="deterministic")
