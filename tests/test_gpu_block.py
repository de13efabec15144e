"""Block and restricted assembly on the GPU against the oracle.

A block form places each sub-form at scalar offsets of one monolithic CSR
matrix / vector (python/cudolfinx/form.py:107-225, assemble.py:112-202); a
restriction drops the dofs outside a given set and numbers the kept ones by
their position in it.  Bar: the monolithic CSR pattern bit-exact with
fe_oracle.block_pattern, values and vectors within the oracle's per-entry
bound (fem_oracle.block_matrix_bound / block_vector_bound), as for single
forms.
"""
import numpy as np
import pytest

from conftest import ensure_library
from gpu_util import tolerance_check
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


def _setup(n=3, seed=9, kind="p2"):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    P = fo.build_problem(kind, n, seed=seed)
    mesh = fem.Mesh(P["coords"], P["cells"], grid_n=n)
    return cx, fem, P, mesh


def test_block_vector_matches_concatenated_vectors():
    # mirrors the reference's test_block_assembly: two P1 spaces, two loads
    cx, fem, P, mesh = _setup(4, 1, "p1")
    V1 = fem.functionspace(mesh, ("P", 1))
    V2 = fem.functionspace(mesh, ("P", 1))
    f1 = fem.Function(V1, P["f"])
    f2 = fem.Function(V2, 1.0 + P["f"] ** 2)
    asm = cx.CUDAAssembler()
    L = cx.form([fem.load(V1, f1), fem.load(V2, f2)])
    assert L.offsets == [0, V1.num_dofs, V1.num_dofs + V2.num_dofs]
    b = asm.create_vector_block(L)
    asm.assemble_vector_block(L, b)
    bh = b.to_host()
    ref, bnd = [], []
    for f in (P["f"], 1.0 + P["f"] ** 2):
        be = fo.p1_load_p1f(P["coords"], P["cells"], f)
        ref.append(fo.assemble_vector(be, P["dofs"], P["ndof"]))
        bnd.append(fo.vector_bound(be, P["dofs"], P["ndof"]))
    ok, worst = tolerance_check(bh, np.concatenate(ref), np.concatenate(bnd))
    assert ok, worst


def _coupled_system(cx, fem, P, mesh, restrict):
    """[[K, -K], [-K, 2K]] on (V, W) (P2, k a P1 field), W restricted to x <= 1/2."""
    V = fem.functionspace(mesh, ("P", 2))
    W = fem.functionspace(mesh, ("P", 2))
    V1 = fem.functionspace(mesh, ("P", 1))
    k = P["k"]
    X = V.tabulate_dof_coordinates()
    R = np.nonzero(X[:, 0] <= 0.5 + 1e-12)[0].astype(np.int32) if restrict else None
    a = [[fem.stiffness(V, fem.Function(V1, k)), fem.stiffness(V, fem.Function(V1, -k), trial=W)],
         [fem.stiffness(W, fem.Function(V1, -k), trial=V), fem.stiffness(W, fem.Function(V1, 2 * k))]]
    g = fem.Function(V, P["g"])
    gW = fem.Function(W, 2.0 * P["g"])
    bcs = [fem.dirichletbc(g, P["bc_dofs"]), fem.dirichletbc(gW, P["bc_dofs"])]
    A = cx.form(a, restriction=([None, R], [None, R]) if restrict else None)
    return A, bcs, R


def _oracle_coupled(P, R):
    dofs, nd = P["dofs"], P["ndof"]
    K = fo.element_matrices(P)
    mk = np.zeros(nd, dtype=np.uint8)
    mk[P["bc_dofs"]] = 1
    if R is None:
        d1, n1, mk1 = dofs, nd, mk
    else:
        d1, n1, mk1 = fo.restricted_dofmap(dofs, R, nd), len(R), mk[R]
    bc1 = np.nonzero(mk1)[0]
    parts = [(dofs, dofs, 1, 1, 0, 0), (dofs, d1, 1, 1, 0, nd), (d1, dofs, 1, 1, nd, 0), (d1, d1, 1, 1, nd, nd)]
    rp, col = fo.block_pattern(parts, nd + n1, nd + n1)
    B = [dict(Ae=K, dofs0=dofs, dofs1=dofs, row_offset=0, col_offset=0, markers0=mk, markers1=mk,
              bc_rows=P["bc_dofs"]),
         dict(Ae=-K, dofs0=dofs, dofs1=d1, row_offset=0, col_offset=nd, markers0=mk, markers1=mk1,
              bc_rows=P["bc_dofs"]),
         dict(Ae=-K, dofs0=d1, dofs1=dofs, row_offset=nd, col_offset=0, markers0=mk1, markers1=mk, bc_rows=bc1),
         dict(Ae=2 * K, dofs0=d1, dofs1=d1, row_offset=nd, col_offset=nd, markers0=mk1, markers1=mk1, bc_rows=bc1)]
    for b in B:
        b.update(bs0=1, bs1=1)
    return rp, col, fo.assemble_block_matrix(B, rp, col), fo.block_matrix_bound(B, rp, col)


@pytest.mark.parametrize("restrict", [False, True])
@pytest.mark.parametrize("nested_bcs", [False, True])
def test_coupled_block_matrix_matches_oracle(restrict, nested_bcs):
    cx, fem, P, mesh = _setup(3, 9)
    A, bcs, R = _coupled_system(cx, fem, P, mesh, restrict)
    asm = cx.CUDAAssembler()
    bc_arg = [[bcs, bcs], [bcs, bcs]] if nested_bcs else bcs
    M = asm.assemble_matrix_block(A, bcs=bc_arg)
    M.assemble()
    rp, col = M.sparsity.to_host()
    rp_o, col_o, v_o, bound = _oracle_coupled(P, R)
    assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o)
    ok, worst = tolerance_check(M.values.cpu().numpy(), v_o, bound)
    assert ok, worst
    # re-assembly into the same matrix (zero=True) reproduces the values
    asm.assemble_matrix_block(A, M, bcs=bc_arg)
    ok, worst = tolerance_check(M.values.cpu().numpy(), v_o, bound)
    assert ok, worst


@pytest.mark.parametrize("kind,bs", [("p2", 1), ("vp2", 3)])
def test_restricted_form_with_lifting_and_set_bc(kind, bs):
    cx, fem, P, mesh = _setup(3, 4, kind)
    nd = P["ndof"]
    if kind == "p2":
        V = fem.functionspace(mesh, ("P", 2))
        V1 = fem.functionspace(mesh, ("P", 1))
        W = fem.functionspace(mesh, ("DG", 0))
        a = fem.stiffness(V, fem.Function(V1, P["k"]))
        L = fem.load(V, fem.Function(W, P["f"]))
        X = V.tabulate_dof_coordinates()
    else:
        V = fem.functionspace(mesh, ("P", 2, (3,)))
        W = fem.functionspace(mesh, ("DG", 0))
        a = fem.elasticity(V, fem.Function(W, P["lam"]), fem.Function(W, P["mu"]))
        W3 = fem.functionspace(mesh, ("DG", 0, (3,)))
        L = fem.load(V, fem.Function(W3, np.asarray(P["f"]).reshape(-1)))
        X = fem.functionspace(mesh, ("P", 2)).tabulate_dof_coordinates()
    R = np.nonzero(X[:, 0] <= 0.5 + 1e-12)[0].astype(np.int32)
    g = np.asarray(P["g"], dtype=np.float64) + 0.25
    bc = fem.dirichletbc(fem.Function(V, g), P["bc_dofs"])
    asm = cx.CUDAAssembler()
    ar = cx.form(a, restriction=[R, R])
    Lr = cx.form(L, restriction=[R])
    A = asm.assemble_matrix(ar, bcs=[bc])
    A.assemble()
    b = asm.assemble_vector(Lr)
    asm.apply_lifting(b, [ar], [[bc]])
    asm.set_bc(b, [bc], V, restriction=R)
    # oracle: restricted numbering, BC markers of the kept dofs
    dr = fo.restricted_dofmap(P["dofs"], R, nd)
    keep = (R.astype(np.int64)[:, None] * bs + np.arange(bs)).ravel()
    mk = np.zeros(nd * bs, dtype=np.uint8)
    mk[P["bc_dofs"]] = 1
    mkr = mk[keep]
    bcr = np.nonzero(mkr)[0]
    nr = len(keep)
    Ae = fo.element_matrices(P)
    rp_o, col_o = fo.block_pattern([(dr, dr, bs, bs, 0, 0)], nr, nr)
    blk = [dict(Ae=Ae, dofs0=dr, dofs1=dr, bs0=bs, bs1=bs, row_offset=0, col_offset=0, markers0=mkr,
                markers1=mkr, bc_rows=bcr)]
    v_o = fo.assemble_block_matrix(blk, rp_o, col_o)
    rp, col = A.sparsity.to_host()
    assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o)
    ok, worst = tolerance_check(A.values.cpu().numpy(), v_o, fo.block_matrix_bound(blk, rp_o, col_o))
    assert ok, worst
    # b = assemble - A_noBC[:, bc] g[bc], then b[bc] = g[bc]
    import scipy.sparse as sp
    v_nobc = fo.assemble_block_matrix([dict(Ae=Ae, dofs0=dr, dofs1=dr, bs0=bs, bs1=bs, row_offset=0,
                                            col_offset=0)], rp_o, col_o)
    An = sp.csr_matrix((v_nobc, col_o, rp_o), shape=(nr, nr))
    gr = g[keep] * mkr
    be = fo.element_vectors(P)
    b_o = fo.assemble_block_vector([(be, dr, bs, 0)], nr) - An @ gr
    b_o[bcr] = g[keep][bcr]
    b_bound = fo.block_vector_bound([(be, dr, bs, 0)], nr) + fo.lifting_bound(nr, Ae, dr, dr, mkr, g[keep], None,
                                                                              1.0, bs, bs)
    b_bound[bcr] = 0.0
    ok, worst = tolerance_check(b.to_host(), b_o, b_bound)
    assert ok, worst


def test_block_forms_reject_other_variants_and_restricted_facets():
    cx, fem, P, mesh = _setup(2, 1)
    A, bcs, R = _coupled_system(cx, fem, P, mesh, True)
    asm = cx.CUDAAssembler()
    M = asm.create_matrix_block(A)
    for variant in ("deterministic", "sorted-slot", "tile", "block"):
        with pytest.raises(RuntimeError, match="atomic scatter only"):
            asm.assemble_matrix(A.forms[0][0], M, variant=variant)
    V = fem.functionspace(mesh, ("P", 2))
    with pytest.raises(RuntimeError, match="unrestricted"):
        cx.form(fem.facet_mass(V, 1.0), restriction=[R, R])


def test_block_matrix_takes_a_packed_bc_collection():
    cx, fem, P, mesh = _setup(2, 3)
    A, bcs, R = _coupled_system(cx, fem, P, mesh, True)
    asm = cx.CUDAAssembler()
    M1 = asm.assemble_matrix_block(A, bcs=bcs)
    M2 = asm.assemble_matrix_block(A, bcs=asm.pack_bcs(bcs))
    M1.assemble()
    M2.assemble()
    # both lie within the oracle's bound of the oracle's values
    _, _, v_o, bound = _oracle_coupled(P, R)
    for M in (M1, M2):
        ok, worst = tolerance_check(M.values.cpu().numpy(), v_o, bound)
        assert ok, worst
