"""Interior-facet (dS) integrals of discontinuous spaces on the GPU against
the oracle: jump penalty on DG0 / DG1 (pattern bit-exact, values within the
oracle's per-entry bound, fem_oracle.matrix_bound), average loads with lifting and
set_bc, the jump-norm functional (1e-12 relative), and a DG cell term plus
its jump term summed into one matrix on the union pattern.

The oracle evaluates both cells' traces at a facet quadrature rule by
barycentric coordinates; the kernels use the closed-form facet integrals and
match the facet's vertices by global index, so the two are independent.
"""
import numpy as np
import pytest

from conftest import ensure_library
from gpu_util import tolerance_check
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


def _mesh(n=3, jitter=0.2, seed=1):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    coords, cells = fo.unit_cube_tet_mesh(n, jitter=jitter, seed=seed)
    mesh = fem.Mesh(coords, cells, grid_n=n)
    return cx, fem, mesh, coords, cells, fo.interior_facets(cells)


@pytest.mark.parametrize("degree", [0, 1])
@pytest.mark.parametrize("alpha_kind", ["constant", "dg0"])
def test_jump_penalty_matches_oracle(degree, alpha_kind):
    cx, fem, mesh, coords, cells, q = _mesh(3, seed=degree)
    C = len(cells)
    V = fem.functionspace(mesh, ("DG", degree))
    assert np.array_equal(fem.interior_facets(mesh), q)
    rng = np.random.default_rng(7)
    if alpha_kind == "constant":
        alpha, af = 2.5, np.full(len(q), 2.5)
    else:
        av = rng.uniform(0.5, 2.0, C)
        alpha, af = fem.Function(fem.functionspace(mesh, ("DG", 0)), av), fo.facet_average(av, q)
    asm = cx.CUDAAssembler()
    a = cx.form(fem.jump_penalty(V, alpha))
    A = asm.assemble_matrix(a)
    A.assemble()
    d = fo.dg_dofmap(C, degree)
    m = fo.macro_dofmap(d, q)
    rp_o, col_o = fo.sparsity(m, m, V.num_dofs)
    Ae = fo.interior_jump_tensors(coords, cells, q, degree, af)
    v_o = fo.assemble_matrix(Ae, m, m, rp_o, col_o)
    rp, col = A.sparsity.to_host()
    assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o)
    ok, worst = tolerance_check(A.values.cpu().numpy(), v_o, fo.matrix_bound(Ae, m, m, rp_o, col_o))
    assert ok, worst


@pytest.mark.parametrize("degree", [0, 1])
def test_average_load_lifting_and_set_bc(degree):
    cx, fem, mesh, coords, cells, q = _mesh(3, seed=3)
    C = len(cells)
    V = fem.functionspace(mesh, ("DG", degree))
    rng = np.random.default_rng(11)
    gv = rng.uniform(-1, 1, C)
    N = V.num_dofs
    bc_dofs = np.sort(rng.choice(N, size=N // 7, replace=False)).astype(np.int32)
    gbc = rng.standard_normal(N)
    bc = fem.dirichletbc(fem.Function(V, gbc), bc_dofs)
    asm = cx.CUDAAssembler()
    a = cx.form(fem.jump_penalty(V, 1.5))
    L = cx.form(fem.facet_average_load(V, fem.Function(fem.functionspace(mesh, ("DG", 0)), gv)))
    b = asm.assemble_vector(L)
    asm.apply_lifting(b, [a], [[bc]])
    asm.set_bc(b, [bc], V)
    d = fo.dg_dofmap(C, degree)
    m = fo.macro_dofmap(d, q)
    be = fo.interior_avg_load(coords, cells, q, degree, fo.facet_average(gv, q))
    b_o = fo.assemble_vector(be, m, N)
    mk = np.zeros(N, dtype=np.uint8)
    mk[bc_dofs] = 1
    Ae = fo.interior_jump_tensors(coords, cells, q, degree, np.full(len(q), 1.5))
    b_o = fo.apply_lifting(b_o, Ae, m, m, mk, gbc)
    b_o = fo.set_bc(b_o, bc_dofs, gbc)
    bound = fo.vector_bound(be, m, N) + fo.lifting_bound(N, Ae, m, m, mk, gbc)
    bound[bc_dofs] = 0.0
    ok, worst = tolerance_check(b.to_host(), b_o, bound)
    assert ok, worst


def test_jump_norm_matches_oracle_and_vanishes_for_continuous_fields():
    cx, fem, mesh, coords, cells, q = _mesh(4, seed=2)
    C = len(cells)
    asm = cx.CUDAAssembler()
    rng = np.random.default_rng(5)
    for degree in (0, 1):
        V = fem.functionspace(mesh, ("DG", degree))
        u = rng.standard_normal(V.num_dofs)
        val = asm.assemble_scalar(cx.form(fem.jump_norm(fem.Function(V, u))))
        ref = fo.interior_jump_norm(coords, cells, q, degree, u[fo.macro_dofmap(fo.dg_dofmap(C, degree), q)])
        assert abs(val - ref) <= 1e-12 * ref
    V1 = fem.functionspace(mesh, ("P", 1))
    val = asm.assemble_scalar(cx.form(fem.jump_norm(fem.Function(V1, rng.standard_normal(V1.num_dofs)))))
    assert val == 0.0


def test_cell_and_jump_terms_in_one_matrix():
    # broken P1 stiffness on DG1 plus the jump penalty: union pattern, summed values
    cx, fem, mesh, coords, cells, q = _mesh(3, seed=4)
    C = len(cells)
    V = fem.functionspace(mesh, ("DG", 1))
    asm = cx.CUDAAssembler()
    # stiffness() wants a Lagrange space: the broken gradient term is the P1
    # stiffness kernel on the DG1 dofmap
    from cudolfinx.fem import FormSpec
    a_cell = cx.form(FormSpec("P1_STIFFNESS", V, [1.0], 2))
    a_jump = cx.form(fem.jump_penalty(V, 4.0))
    A = asm.create_matrix([a_cell, a_jump])
    asm.assemble_matrix(a_cell, A)
    asm.assemble_matrix(a_jump, A, zero=False)
    A.assemble()
    d = fo.dg_dofmap(C, 1)
    m = fo.macro_dofmap(d, q)
    N = V.num_dofs
    rp_o, col_o = fo.block_pattern([(d, d, 1, 1, 0, 0), (m, m, 1, 1, 0, 0)], N, N)
    blk = [dict(Ae=fo.p1_stiffness(coords, cells), dofs0=d, dofs1=d, bs0=1, bs1=1, row_offset=0, col_offset=0),
           dict(Ae=fo.interior_jump_tensors(coords, cells, q, 1, np.full(len(q), 4.0)), dofs0=m, dofs1=m, bs0=1,
                bs1=1, row_offset=0, col_offset=0)]
    v_o = fo.assemble_block_matrix(blk, rp_o, col_o)
    rp, col = A.sparsity.to_host()
    assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o)
    ok, worst = tolerance_check(A.values.cpu().numpy(), v_o, fo.block_matrix_bound(blk, rp_o, col_o))
    assert ok, worst


def test_interior_facet_errors():
    cx, fem, mesh, coords, cells, q = _mesh(2)
    V = fem.functionspace(mesh, ("DG", 1))
    bad = q.copy()
    bad[0, 3] = (bad[0, 3] + 1) % 4  # the second side names another facet of its cell
    with pytest.raises(RuntimeError, match="different triangles"):
        cx.form(fem.jump_penalty(V, 1.0, facets=bad))
    asm = cx.CUDAAssembler()
    a = cx.form(fem.jump_penalty(V, 1.0))
    A = asm.create_matrix(a)
    for variant in ("deterministic", "tile", "block"):
        with pytest.raises(RuntimeError, match="atomic scatter only"):
            asm.assemble_matrix(a, A, variant=variant)
