"""Diagonal of a bilinear form assembled as a vector (the reference's
test_diagonal_assembly, python/test/test_cuda_assembly.py:199-208: a form
compiled with form_compiler_options={"part": "diagonal"} and assembled with
assemble_vector).

Checked against the oracle's diagonal (FP64: within the per-entry bound
fem_oracle.diagonal_bound, atomics add in another order), the diagonal slots of the
matrix the engine assembles without BCs, and for FP32 element tensors at the
FP32 level (relative 2-norm error below 2e-6).
"""
import numpy as np
import pytest

from conftest import ensure_library
from gpu_util import mirror_problem, tolerance_check
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,n", [("p1", 6), ("p1k", 7), ("p2", 5), ("p3", 3), ("vp2", 3)])
def test_diagonal_matches_the_oracle_and_the_matrix_diagonal(kind, n):
    P = fo.build_problem(kind, n, seed=11)
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    d_form = cx.form(M["a"], form_compiler_options={"part": "diagonal"})
    assert d_form.rank == 1 and d_form.part == "diagonal"
    d = asm.assemble_vector(d_form).to_host()
    nscal = P["ndof"] * P["bs"]
    assert d.shape == (nscal,)
    Ae = fo.element_matrices(P)
    ref = fo.assemble_diagonal(Ae, P["dofs"], nscal, P["bs"])
    bound = fo.diagonal_bound(Ae, P["dofs"], nscal, P["bs"])
    ok, worst = tolerance_check(d, ref, bound)
    assert ok, worst
    # the same numbers as the diagonal slots of A assembled without BCs
    a = cx.form(M["a"])
    A = asm.assemble_matrix(a)
    A.assemble()
    rp, col = A.sparsity.to_host()
    diag = A.values.cpu().numpy()[fo.diag_positions(rp, col)]
    ok, worst = tolerance_check(diag, ref, bound)
    assert ok, worst
    # accumulate into an existing vector: zero=False adds
    v = asm.create_vector(d_form)
    asm.assemble_vector(d_form, v)
    asm.assemble_vector(d_form, v, zero=False)
    ok, worst = tolerance_check(v.to_host(), 2.0 * ref, 2.0 * bound)
    assert ok, worst


@pytest.mark.parametrize("kind,n", [("p2", 5), ("p3", 3), ("vp2", 3)])
def test_fp32_diagonal_at_fp32_level(kind, n):
    P = fo.build_problem(kind, n, seed=12)
    M = mirror_problem(P, precision="fp32")
    cx = M["cx"]
    d = cx.CUDAAssembler().assemble_vector(cx.form(M["a"], form_compiler_options={"part": "diagonal"})).to_host()
    ref = fo.assemble_diagonal(fo.element_matrices(P), P["dofs"], P["ndof"] * P["bs"], P["bs"])
    rel = np.linalg.norm(d - ref) / np.linalg.norm(ref)
    assert 0.0 < rel < 2e-6, rel


def test_restricted_diagonal_is_the_kept_part():
    P = fo.build_problem("p2", 4, seed=13)
    M = mirror_problem(P)
    cx = M["cx"]
    rng = np.random.default_rng(0)
    keep = np.sort(rng.choice(P["ndof"], size=P["ndof"] // 2, replace=False)).astype(np.int32)
    f = cx.form(M["a"], restriction=[keep], form_compiler_options={"part": "diagonal"})
    d = cx.CUDAAssembler().assemble_vector(f).to_host()
    Ae = fo.element_matrices(P)
    full = fo.assemble_diagonal(Ae, P["dofs"], P["ndof"])
    bound = fo.diagonal_bound(Ae, P["dofs"], P["ndof"])
    assert d.shape == (len(keep),)
    ok, worst = tolerance_check(d, full[keep], bound[keep])
    assert ok, worst


def test_diagonal_part_rejects_linear_facet_and_mixed_forms():
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    mesh = fem.create_unit_cube(2)
    V = fem.functionspace(mesh, ("P", 2))
    V1 = fem.functionspace(mesh, ("P", 1))
    opts = {"form_compiler_options": {"part": "diagonal"}}
    with pytest.raises(ValueError):
        cx.form(fem.load(V, 1.0), **opts)
    with pytest.raises(ValueError):
        cx.form(fem.facet_mass(V1, 1.0, fem.exterior_facets(mesh)), **opts)
    with pytest.raises(ValueError):
        cx.form(fem.stiffness(V, 1.0), form_compiler_options={"part": "lower"})
    V2 = fem.functionspace(mesh, ("P", 2))  # a second field: another space
    with pytest.raises(ValueError):
        cx.form(fem.stiffness(V, 1.0, trial=V2), **opts)
