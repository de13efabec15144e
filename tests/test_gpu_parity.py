"""GPU parity: the CUDA path (through the C-ABI) against the CPU oracle.

Bar: identical CSR pattern (bit-exact); CSR values and right-hand sides in
FP64 within the oracle's per-entry bound: 1e-12 times the sum of the entry's
|contributions| plus 1e-14 times each contributing element's largest |entry|
(no floor relative to the whole matrix), and exact where set_diagonal /
set_bc write; the deterministic variant is also bitwise reproducible from
run to run.
"""
import glob
import os

import numpy as np
import pytest

from gpu_util import mirror_problem, run_system, tolerance_check
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# p1k: DG0 k log-uniform over 1e-2..1e2, so cells of four decades meet in
# one block of the block variant
CASES = [("p1", 2), ("p1", 7), ("p1", 16), ("p1k", 6), ("p1k", 12), ("p2", 2), ("p2", 5), ("p2", 9), ("vp2", 2),
         ("vp2", 4), ("p3", 2), ("p3", 4)]


def _problem_from_golden(path):
    G = np.load(path)
    kind = os.path.basename(path).split("_n")[0]
    P = {"kind": kind, "n": int(G["n"]), "coords": G["coords"], "cells": G["cells"], "dofs": G["dofs"],
         "bc_dofs": G["bc_dofs"], "g": G["g"], "ndof": int(G["ndof"]), "bs": int(G["bs"])}
    for k in ("k", "f", "lam", "mu"):
        P[k] = G[k] if k in G.files else None
    return P, G


VARIANTS = ["auto", "atomic", "atomic-full", "tile", "deterministic", "sorted-slot", "row-gather", "block", "grouped",
            "coalesced"]


def _supported(kind, variant):
    if variant == "row-gather":
        return kind in ("p1", "p1k")
    if variant == "grouped":
        return kind == "p2"
    if variant == "coalesced":
        return kind in ("p2", "vp2", "p3")
    if variant in ("tile", "block"):
        return kind in ("p1", "p1k", "p2")
    return True


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
@pytest.mark.parametrize("variant", VARIANTS)
def test_golden_fixtures(path, variant):
    P, G = _problem_from_golden(path)
    if not _supported(P["kind"], variant):
        pytest.skip("variant not offered for this element")
    R = run_system(P, variant=variant)
    assert np.array_equal(R["row_ptr"], G["row_ptr"]) and np.array_equal(R["col"], G["col"])
    ok, worst = tolerance_check(R["A"], G["A"], G["A_bound"])
    assert ok, worst
    ok, worst = tolerance_check(R["b"], G["b"], G["b_bound"])
    assert ok, worst


@pytest.mark.parametrize("kind,n", CASES)
@pytest.mark.parametrize("variant", VARIANTS)
def test_system_parity(kind, n, variant):
    if not _supported(kind, variant):
        pytest.skip("variant not offered for this element")
    P = fo.build_problem(kind, n, seed=n)
    S = fo.solve_system(P)
    R = run_system(P, variant=variant)
    assert np.array_equal(R["row_ptr"], S["row_ptr"]) and np.array_equal(R["col"], S["col"])
    ok, worst = tolerance_check(R["A"], S["A"], S["A_bound"])
    assert ok, f"A: worst error / bound {worst}"
    ok, worst = tolerance_check(R["b"], S["b"], S["b_bound"])
    assert ok, f"b: worst error / bound {worst}"


@pytest.mark.parametrize("kind,n,variant", [("p1", 8, "deterministic"), ("p2", 5, "deterministic"),
                                            ("p1", 8, "sorted-slot"), ("vp2", 3, "deterministic"),
                                            ("p3", 3, "deterministic")])
def test_deterministic_is_bitwise_reproducible(kind, n, variant):
    P = fo.build_problem(kind, n, seed=3)
    R1 = run_system(P, variant=variant)
    asm, A, (a, _), bcs = R1["asm"], R1["Aobj"], R1["forms"], R1["bcs"]
    first = A.values.clone()
    for _ in range(3):
        asm.assemble_matrix(a, A, bcs=bcs, variant=variant)
        A.assemble()
        assert bool((A.values == first).all())


def test_matrix_without_bcs_and_zero_false_accumulates():
    P = fo.build_problem("p2", 4, seed=1)
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    a = cx.form(M["a"])
    A = asm.assemble_matrix(a)
    A.assemble()
    Ae = fo.element_matrices(P)
    rp, col = fo.sparsity(P["dofs"], P["dofs"], P["ndof"])
    ref = fo.assemble_matrix(Ae, P["dofs"], P["dofs"], rp, col)
    bound = fo.matrix_bound(Ae, P["dofs"], P["dofs"], rp, col)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref, bound)
    assert ok, worst
    for variant in ("atomic", "tile", "deterministic", "sorted-slot"):
        asm.assemble_matrix(a, A, zero=False, variant=variant)
        A.assemble()
    # five assemblies summed: five times the contributions
    ok, worst = tolerance_check(A.values.cpu().numpy(), 5 * ref, 5 * bound)
    assert ok, worst


def test_reassembly_after_coefficient_update():
    # the reference's test_reassembly: change a coefficient on the host, re-assemble
    P = fo.build_problem("p2", 4, seed=2)
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    L = cx.form(M["L"])
    fL = M["L"].coefficients[0]
    b = asm.assemble_vector(L)
    for d in (2.0, 3.0):
        fL.x.array[:] = P["f"] * d
        asm.assemble_vector(L, b)
        be = fo.p2_load_dg0(P["coords"], P["cells"], P["f"] * d)
        ref = fo.assemble_vector(be, P["dofs"], P["ndof"])
        ok, worst = tolerance_check(b.to_host(), ref, fo.vector_bound(be, P["dofs"], P["ndof"]))
        assert ok, worst


def test_lifting_with_x0_and_scale():
    P = fo.build_problem("p2", 4, seed=4)
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    a, L = cx.form(M["a"]), cx.form(M["L"])
    bcs = asm.pack_bcs([M["bc"]])
    rng = np.random.default_rng(0)
    x0h = rng.standard_normal(P["ndof"])
    x0 = asm.create_vector(L)
    import torch
    x0.vector.copy_(torch.from_numpy(x0h))
    b = asm.assemble_vector(L)
    asm.apply_lifting(b, [a], [bcs], x0=[x0], scale=-0.7)
    asm.set_bc(b, bcs, M["V"], x0=x0, scale=-0.7)
    markers = np.zeros(P["ndof"], np.uint8)
    markers[P["bc_dofs"]] = 1
    be, Ae = fo.element_vectors(P), fo.element_matrices(P)
    ref = fo.assemble_vector(be, P["dofs"], P["ndof"])
    ref = fo.apply_lifting(ref, Ae, P["dofs"], P["dofs"], markers, P["g"], x0h, -0.7)
    ref = fo.set_bc(ref, P["bc_dofs"], P["g"], x0h, -0.7)
    bound = fo.vector_bound(be, P["dofs"], P["ndof"]) + fo.lifting_bound(P["ndof"], Ae, P["dofs"], P["dofs"],
                                                                          markers, P["g"], x0h, -0.7)
    bound[P["bc_dofs"]] = 0.0
    ok, worst = tolerance_check(b.to_host(), ref, bound)
    assert ok, worst


@pytest.mark.parametrize("kind,n", [("p1", 6), ("p1k", 5), ("p2", 4), ("vp2", 3), ("p3", 3)])
def test_fused_rhs_matches_the_three_calls(kind, n):
    # fe_assemble_rhs (vector + lifting + set_bc in one kernel) against the
    # oracle under its bound, and against the three calls: BC rows equal
    import torch

    P = fo.build_problem(kind, n, seed=11)
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    a, L = cx.form(M["a"]), cx.form(M["L"])
    bcs = asm.pack_bcs([M["bc"]])
    bs = P["bs"]
    nscal = P["ndof"] * bs
    x0h = np.random.default_rng(1).standard_normal(nscal)
    x0 = asm.create_vector(L)
    x0.vector.copy_(torch.from_numpy(x0h))
    fused = asm.assemble_rhs(L, a, bcs, x0=x0, scale=-0.7)
    b3 = asm.assemble_vector(L)
    asm.apply_lifting(b3, [a], [bcs], x0=[x0], scale=-0.7)
    asm.set_bc(b3, bcs, M["V"], x0=x0, scale=-0.7)
    markers = np.zeros(nscal, np.uint8)
    markers[P["bc_dofs"]] = 1
    be, Ae = fo.element_vectors(P), fo.element_matrices(P)
    dofs = P["dofs"]
    ref = fo.assemble_vector(be, dofs, nscal, bs)
    ref = fo.apply_lifting(ref, Ae, dofs, dofs, markers, P["g"], x0h, -0.7, bs, bs)
    ref = fo.set_bc(ref, P["bc_dofs"], P["g"], x0h, -0.7)
    bound = fo.vector_bound(be, dofs, nscal, bs) + fo.lifting_bound(nscal, Ae, dofs, dofs, markers, P["g"], x0h,
                                                                    -0.7, bs, bs)
    bound[P["bc_dofs"]] = 0.0
    out, out3 = fused.to_host(), b3.to_host()
    ok, worst = tolerance_check(out, ref, bound)
    assert ok, worst
    assert np.array_equal(out[P["bc_dofs"]], out3[P["bc_dofs"]])
    ok, worst = tolerance_check(out, out3, 2 * bound)
    assert ok, worst
    # re-assembly into the same vector (zero=True) gives the same values again
    asm.assemble_rhs(L, a, bcs, vec=fused, x0=x0, scale=-0.7)
    ok, worst = tolerance_check(fused.to_host(), ref, bound)
    assert ok, worst


def test_fused_rhs_without_bcs_is_the_vector():
    P = fo.build_problem("p2", 3, seed=12)
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    a, L = cx.form(M["a"]), cx.form(M["L"])
    out = asm.assemble_rhs(L, a, []).to_host()
    be = fo.element_vectors(P)
    ref = fo.assemble_vector(be, P["dofs"], P["ndof"])
    ok, worst = tolerance_check(out, ref, fo.vector_bound(be, P["dofs"], P["ndof"]))
    assert ok, worst


def test_bc_update_changes_values_not_pattern():
    P = fo.build_problem("p2", 3, seed=5)
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    L = cx.form(M["L"])
    bcs = asm.pack_bcs([M["bc"]])
    b = asm.assemble_vector(L)
    M["bc"].value.x.array[:] *= 2.0
    bcs.update()
    asm.set_bc(b, bcs, M["V"])
    out = b.to_host()
    assert np.allclose(out[P["bc_dofs"]], 2.0 * P["g"][P["bc_dofs"]], rtol=1e-15, atol=0)


def test_fp32_element_tensors_precision_path():
    # FP32 contraction, FP64 accumulation: relative Frobenius error at FP32 level
    for kind, n in (("p2", 6), ("vp2", 3), ("p3", 3)):
        P = fo.build_problem(kind, n, seed=6)
        S = fo.solve_system(P)
        R = run_system(P, precision="fp32")
        rel = np.linalg.norm(R["A"] - S["A"]) / np.linalg.norm(S["A"])
        assert rel < 2e-6, (kind, rel)
        assert rel > 0.0


def test_pcg_solution_matches_direct_solve():
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    for kind, n in (("p1", 8), ("p2", 5), ("vp2", 3), ("p3", 3)):
        P = fo.build_problem(kind, n, seed=7)
        R = run_system(P)
        N = len(R["row_ptr"]) - 1
        A = sp.csr_matrix((R["A"], R["col"], R["row_ptr"]), shape=(N, N))
        x_ref = spla.spsolve(A.tocsc(), R["b"])
        x, it, res = R["asm"].solve(R["Aobj"], R["bobj"], rtol=1e-10)
        xh = x.to_host()
        assert res <= 1e-10 and it > 0
        assert np.linalg.norm(xh - x_ref) <= 1e-7 * np.linalg.norm(x_ref)


def test_mixed_precision_pcg_meets_rtol_in_fp64():
    # inner iterations on FP32 values (block size 3: 3x3 block columns),
    # refined in FP64: the FP64 residual meets rtol and x matches a direct solve
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    for kind, n, bs in (("p2", 5, 1), ("vp2", 3, 3), ("p1", 8, 1)):
        P = fo.build_problem(kind, n, seed=9)
        R = run_system(P)
        N = len(R["row_ptr"]) - 1
        A = sp.csr_matrix((R["A"], R["col"], R["row_ptr"]), shape=(N, N))
        x_ref = spla.spsolve(A.tocsc(), R["b"])
        x, it, res = R["asm"].solve(R["Aobj"], R["bobj"], rtol=1e-10, precision="mixed", block_size=bs)
        xh = x.to_host()
        assert res <= 1e-10 and it > 0
        assert np.linalg.norm(A @ xh - R["b"]) <= 1.5e-10 * np.linalg.norm(R["b"])
        assert np.linalg.norm(xh - x_ref) <= 1e-7 * np.linalg.norm(x_ref)
    # a scalar pattern is not block-structured
    P = fo.build_problem("p2", 3, seed=9)
    R = run_system(P)
    with pytest.raises(RuntimeError, match="block size 3"):
        R["asm"].solve(R["Aobj"], R["bobj"], precision="mixed", block_size=3)


def test_pcg_reports_non_convergence():
    P = fo.build_problem("p2", 5, seed=8)
    R = run_system(P)
    x, it, res = R["asm"].solve(R["Aobj"], R["bobj"], rtol=1e-12, max_iter=3, raise_on_failure=False)
    assert it == 3 and res > 1e-12
    with pytest.raises(RuntimeError, match="PCG stopped"):
        R["asm"].solve(R["Aobj"], R["bobj"], rtol=1e-12, max_iter=3)


def test_missing_coupling_is_reported_not_faulted():
    # a pattern without the off-diagonal couplings: binding reports FE_ERR_PATTERN
    P = fo.build_problem("p1", 2, seed=0)
    M = mirror_problem(P)
    cx = M["cx"]
    a = cx.form(M["a"])
    n = P["ndof"]
    rp = np.arange(n + 1, dtype=np.int32)
    col = np.arange(n, dtype=np.int32)
    ctx = cx.get_cuda_context()
    sp_diag = cx.Sparsity.from_csr(ctx, rp, col, n)
    with pytest.raises(RuntimeError, match="coupling missing"):
        a._bind(sp_diag)
    # the context stays usable afterwards
    asm = cx.CUDAAssembler()
    A = asm.assemble_matrix(cx.form(M["a"]))
    A.assemble()


def test_empty_bc_and_empty_mesh():
    import cudolfinx as cx
    from cudolfinx import fem

    m = fem.Mesh(np.zeros((0, 3)), np.zeros((0, 4), np.int32))
    V = fem.functionspace(m, ("P", 1))
    asm = cx.CUDAAssembler()
    a = cx.form(fem.stiffness(V))
    A = asm.assemble_matrix(a, bcs=[])
    A.assemble()
    assert A.sparsity.nnz == 0


@pytest.mark.parametrize("variant", ["grouped", "coalesced"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_grouped_variant_on_permuted_cells_and_renumbered_dofs(precision, variant):
    # the grouped plan comes from the dofmap and the cell centroids only: a
    # random cell order and a random dof numbering give the same matrix
    from conftest import ensure_library
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    n = 7
    P = fo.build_problem("p2", n, seed=21)
    rng = np.random.default_rng(5)
    cp = rng.permutation(len(P["cells"]))
    cells = P["cells"][cp]
    mesh = fem.Mesh(P["coords"], cells, grid_n=n)
    V = fem.functionspace(mesh, ("P", 2))
    dp = rng.permutation(V.num_nodes).astype(np.int32)  # new number of each dof
    V.dofs = np.ascontiguousarray(dp[V.dofs])
    V1 = fem.functionspace(mesh, ("P", 1))
    k = fem.Function(V1, P["k"])
    bdofs = np.sort(dp[P["bc_dofs"]]).astype(np.int32)
    g = np.zeros(V.num_dofs)
    g[dp] = P["g"]
    bc = fem.dirichletbc(fem.Function(V, g), bdofs)
    asm = cx.CUDAAssembler()
    a = cx.form(fem.stiffness(V, k, precision=precision))
    A = asm.assemble_matrix(a, bcs=[bc], variant=variant)
    A.assemble()
    rp, col = A.sparsity.to_host()
    rp_o, col_o = fo.sparsity(V.dofs, V.dofs, V.num_nodes)
    assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o)
    Ae = fo.p2_stiffness(P["coords"], cells, P["k"][cells])
    mk = np.zeros(V.num_dofs, dtype=np.uint8)
    mk[bdofs] = 1
    ref = fo.assemble_matrix(Ae, V.dofs, V.dofs, rp_o, col_o, 1, 1, mk, mk, 1.0, bdofs)
    if precision == "fp64":
        ok, worst = tolerance_check(A.values.cpu().numpy(), ref,
                                    fo.matrix_bound(Ae, V.dofs, V.dofs, rp_o, col_o, 1, 1, mk, mk))
        assert ok, worst
    else:
        rel = np.linalg.norm(A.values.cpu().numpy() - ref) / np.linalg.norm(ref)
        assert 0.0 < rel < 2e-6, rel


@pytest.mark.parametrize("kind", ["p1", "p2"])
@pytest.mark.parametrize("shape", [(32, 1), (64, 1), (128, 1), (64, 0), (128, 0)])
def test_atomic_launch_shapes(kind, shape):
    # the tuner's launch shapes of the atomic scatter (cells per CTA, byte-map staging)
    from cudolfinx import _lib

    if kind == "p1" and shape[1] == 0:
        pytest.skip("the P1 kernel reads its byte map directly in every shape")
    P = fo.build_problem(kind, 5, seed=17)
    S = fo.solve_system(P)
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    a = cx.form(M["a"])
    _lib.check(_lib.lib.fe_form_set_launch(a.cuda_form, *shape), "fe_form_set_launch")
    A = asm.assemble_matrix(a, bcs=asm.pack_bcs([M["bc"]]), variant="atomic-full")
    A.assemble()
    ok, worst = tolerance_check(A.values.cpu().numpy(), S["A"], S["A_bound"])
    assert ok, worst
    with pytest.raises(RuntimeError, match="cells per CTA"):
        _lib.check(_lib.lib.fe_form_set_launch(a.cuda_form, 48, 1), "fe_form_set_launch")


def test_coalesced_p3_on_permuted_cells_and_renumbered_dofs():
    # the coalesced P3 kernel (FP64 default) reads each cell's slot bytes as
    # words from the byte map: a random cell order and dof numbering give the
    # oracle's matrix for that numbering
    from conftest import ensure_library
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    n = 5
    P = fo.build_problem("p3", n, seed=29)
    rng = np.random.default_rng(7)
    cp = rng.permutation(len(P["cells"]))
    cells = P["cells"][cp]
    mesh = fem.Mesh(P["coords"], cells, grid_n=n)
    V = fem.functionspace(mesh, ("P", 3))
    dp = rng.permutation(V.num_nodes).astype(np.int32)
    V.dofs = np.ascontiguousarray(dp[V.dofs])
    W = fem.functionspace(mesh, ("DG", 0))
    kc = P["k"][cp]
    k = fem.Function(W, kc)
    bdofs = np.sort(dp[P["bc_dofs"]]).astype(np.int32)
    g = np.zeros(V.num_dofs)
    g[dp] = P["g"]
    bc = fem.dirichletbc(fem.Function(V, g), bdofs)
    asm = cx.CUDAAssembler()
    a = cx.form(fem.stiffness(V, k))
    A = asm.assemble_matrix(a, bcs=[bc], variant="coalesced")
    A.assemble()
    rp, col = A.sparsity.to_host()
    rp_o, col_o = fo.sparsity(V.dofs, V.dofs, V.num_nodes)
    assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o)
    Ae = fo.p3_stiffness(P["coords"], cells, kc)
    mk = np.zeros(V.num_dofs, dtype=np.uint8)
    mk[bdofs] = 1
    ref = fo.assemble_matrix(Ae, V.dofs, V.dofs, rp_o, col_o, 1, 1, mk, mk, 1.0, bdofs)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref,
                                fo.matrix_bound(Ae, V.dofs, V.dofs, rp_o, col_o, 1, 1, mk, mk))
    assert ok, worst


@pytest.mark.parametrize("stage", [1, 0])
def test_coalesced_p2_slot_byte_fetch(stage):
    # the coalesced P2 kernel with its slot bytes staged in shared memory (1)
    # or fetched as words and handed out by shuffles (0), on P2 n=9 (4,374
    # cells: a partial last CTA)
    from cudolfinx import _lib

    P = fo.build_problem("p2", 9, seed=23)
    S = fo.solve_system(P)
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    a = cx.form(M["a"])
    _lib.check(_lib.lib.fe_form_set_launch(a.cuda_form, 64, stage), "fe_form_set_launch")
    A = asm.assemble_matrix(a, bcs=asm.pack_bcs([M["bc"]]), variant="coalesced")
    A.assemble()
    ok, worst = tolerance_check(A.values.cpu().numpy(), S["A"], S["A_bound"])
    assert ok, worst


@pytest.mark.parametrize("kind,n", [("p1", 7), ("p1k", 8)])
@pytest.mark.parametrize("bcs", ["same", "rows-only", "none"])
def test_block_variant_bc_paths(kind, n, bcs):
    # the P1 block kernel with the same BCs on rows and columns, with row BCs
    # only, and with none, against the oracle
    import torch

    from cudolfinx import _lib

    P = fo.build_problem(kind, n, seed=21)
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    a = cx.form(M["a"])
    A = asm.create_matrix(a)
    dbc = asm.pack_bcs([M["bc"]])  # keeps the BC object (and its handle) alive
    hbc = dbc._get_cpp_bcs(M["V"]).handle
    b0, b1 = {"same": (hbc, hbc), "rows-only": (hbc, None), "none": (None, None)}[bcs]
    flags = _lib.ASM_ZERO | _lib.VARIANT_FLAGS["block"]
    _lib.check(_lib.lib.fe_assemble_matrix(a.cuda_form, A.values.data_ptr(), b0, b1, 1.0, flags,
                                           torch.cuda.current_stream().cuda_stream), "block")
    torch.cuda.synchronize()
    rp, col = A.sparsity.to_host()
    mk = np.zeros(P["ndof"], np.uint8)
    mk[P["bc_dofs"]] = 1
    m0 = mk if b0 is not None else None
    m1 = mk if b1 is not None else None
    Ae = fo.element_matrices(P)
    ref = fo.assemble_matrix(Ae, P["dofs"], P["dofs"], rp, col, 1, 1, m0, m1, 1.0,
                             P["bc_dofs"] if b0 is not None else None)
    bound = fo.matrix_bound(Ae, P["dofs"], P["dofs"], rp, col, 1, 1, m0, m1)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref, bound)
    assert ok, worst


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_vp2_coalesced_matches_atomic_and_is_symmetric(precision):
    # the warp-coalesced vector-P2 kernel (default) against the thread-per-cell
    # upper-triangle scatter: same values up to the summation order (FP64) or
    # the FP32 rounding of the element entries; symmetric to rounding level
    import scipy.sparse as sp
    from scipy.sparse.linalg import norm as spnorm

    P = fo.build_problem("vp2", 4, seed=13)
    Rc = run_system(P, precision=precision, variant="coalesced")
    Ra = run_system(P, precision=precision, variant="atomic")
    assert np.array_equal(Rc["row_ptr"], Ra["row_ptr"]) and np.array_equal(Rc["col"], Ra["col"])
    rel = np.linalg.norm(Rc["A"] - Ra["A"]) / np.linalg.norm(Ra["A"])
    assert rel < (1e-14 if precision == "fp64" else 1e-6), rel
    N = len(Rc["row_ptr"]) - 1
    A = sp.csr_matrix((Rc["A"], Rc["col"], Rc["row_ptr"]), shape=(N, N))
    asym = spnorm(A - A.T) / spnorm(A)
    assert asym < 1e-14, asym


@pytest.mark.parametrize("renumber", [False, True])
def test_p2_default_scatter_on_a_larger_mesh(renumber):
    # the default P2 scatter (warp-coalesced) on P2 n=24 (82,944 cells,
    # 1,296 CTAs), in the mesh's order and with a random cell order and dof
    # numbering; assembled twice into the same values, the second time over
    # NaN (the zero pass must reach every slot)
    from conftest import ensure_library
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    n = 24
    P = fo.build_problem("p2", n, seed=17)
    rng = np.random.default_rng(5)
    cells = P["cells"][rng.permutation(len(P["cells"]))] if renumber else P["cells"]
    mesh = fem.Mesh(P["coords"], cells, grid_n=n)
    V = fem.functionspace(mesh, ("P", 2))
    dp = rng.permutation(V.num_nodes).astype(np.int32) if renumber else np.arange(V.num_nodes, dtype=np.int32)
    if renumber:
        V.dofs = np.ascontiguousarray(dp[V.dofs])
    V1 = fem.functionspace(mesh, ("P", 1))
    k = fem.Function(V1, P["k"])
    bdofs = np.sort(dp[P["bc_dofs"]]).astype(np.int32)
    g = np.zeros(V.num_dofs)
    g[dp] = P["g"]
    bc = fem.dirichletbc(fem.Function(V, g), bdofs)
    asm = cx.CUDAAssembler()
    a = cx.form(fem.stiffness(V, k))
    A = asm.assemble_matrix(a, bcs=[bc])
    A.values.fill_(float("nan"))
    asm.assemble_matrix(a, A, bcs=[bc])
    A.assemble()
    assert np.isfinite(A.values.cpu().numpy()).all()
    rp, col = A.sparsity.to_host()
    rp_o, col_o = fo.sparsity(V.dofs, V.dofs, V.num_nodes)
    assert np.array_equal(rp, rp_o) and np.array_equal(col, col_o)
    Ae = fo.p2_stiffness(P["coords"], cells, P["k"][cells])
    mk = np.zeros(V.num_dofs, dtype=np.uint8)
    mk[bdofs] = 1
    ref = fo.assemble_matrix(Ae, V.dofs, V.dofs, rp_o, col_o, 1, 1, mk, mk, 1.0, bdofs)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref,
                                fo.matrix_bound(Ae, V.dofs, V.dofs, rp_o, col_o, 1, 1, mk, mk))
    assert ok, worst
