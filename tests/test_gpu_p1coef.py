"""P1 stiffness with a P1 coefficient field k: the gradients are constant on a
cell, so the entries are exactly mean(k) |det J|/6 grad phi_i . grad phi_j.

Checked against the oracle (within its per-entry bound, fem_oracle.matrix_bound) for
the atomic, full-scatter and deterministic variants with BCs, for lifting and
the diagonal part; "auto" on a mesh above the block kernel's threshold falls
back to the atomic scatter (the block and tile kernels take constant or DG0
coefficients); the variant tuner skips the variants a form is refused by.
"""
import numpy as np
import pytest

from conftest import ensure_library
from gpu_util import tolerance_check
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


def _problem(n, seed):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    P = fo.build_problem("p1", n, seed=seed)
    mesh = fem.Mesh(P["coords"], P["cells"], grid_n=n)
    V = fem.functionspace(mesh, ("P", 1))
    kv = np.exp(np.random.default_rng(seed).standard_normal(len(P["coords"])))
    k = fem.Function(fem.functionspace(mesh, ("P", 1)), kv)
    Ae = fo.p1_stiffness(P["coords"], P["cells"], kv[P["cells"]].mean(axis=1))
    return cx, fem, P, V, k, Ae


@pytest.mark.parametrize("variant", ["auto", "atomic", "atomic-full", "deterministic"])
def test_p1_stiffness_with_p1_coefficient_matches_oracle(variant):
    cx, fem, P, V, k, Ae = _problem(7, 3)
    asm = cx.CUDAAssembler()
    a = cx.form(fem.stiffness(V, k))
    bc = fem.dirichletbc(fem.Function(V, P["g"] + 1.0), P["bc_dofs"])
    bcs = asm.pack_bcs([bc])
    A = asm.assemble_matrix(a, bcs=bcs, variant=variant)
    A.assemble()
    rp, col = A.sparsity.to_host()
    markers = np.zeros(P["ndof"], dtype=np.uint8)
    markers[P["bc_dofs"]] = 1
    ref = fo.assemble_matrix(Ae, P["dofs"], P["dofs"], rp, col, 1, 1, markers, markers, 1.0, P["bc_dofs"])
    bound = fo.matrix_bound(Ae, P["dofs"], P["dofs"], rp, col, 1, 1, markers, markers)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref, bound)
    assert ok, worst
    # lifting with g = 1 + the oracle's g, and the diagonal part
    b = asm.assemble_vector(cx.form(fem.load(V, 0.0)))
    asm.apply_lifting(b, [a], [bcs])
    ok, worst = tolerance_check(b.to_host(), fo.apply_lifting(np.zeros(P["ndof"]), Ae, P["dofs"], P["dofs"],
                                                              markers, P["g"] + 1.0),
                                fo.lifting_bound(P["ndof"], Ae, P["dofs"], P["dofs"], markers, P["g"] + 1.0))
    assert ok, worst
    d = asm.assemble_vector(cx.form(fem.stiffness(V, k), form_compiler_options={"part": "diagonal"})).to_host()
    ok, worst = tolerance_check(d, fo.assemble_diagonal(Ae, P["dofs"], P["ndof"]),
                                fo.diagonal_bound(Ae, P["dofs"], P["ndof"]))
    assert ok, worst


def test_auto_falls_back_to_the_atomic_scatter_on_large_meshes():
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    n = 57  # 1,111,158 cells: above the block kernel's 2^20-cell threshold
    mesh = fem.create_unit_cube(n)
    V = fem.functionspace(mesh, ("P", 1))
    kv = 1.0 + mesh.geometry_x[:, 0]
    k = fem.Function(V, kv)
    asm = cx.CUDAAssembler()
    a = cx.form(fem.stiffness(V, k))
    A1 = asm.assemble_matrix(a, variant="auto")
    A2 = asm.assemble_matrix(a, variant="atomic-full")
    A1.assemble()
    A2.assemble()
    cells = mesh.cells
    Ae = fo.p1_stiffness(mesh.geometry_x, cells, kv[cells].mean(axis=1))
    rp, col = A1.sparsity.to_host()
    ref = fo.assemble_matrix(Ae, V.dofs, V.dofs, rp, col)
    bound = fo.matrix_bound(Ae, V.dofs, V.dofs, rp, col)
    for A in (A1, A2):
        ok, worst = tolerance_check(A.values.cpu().numpy(), ref, bound)
        assert ok, worst
    with pytest.raises(RuntimeError):
        asm.assemble_matrix(a, variant="block")
    # the tuner skips the refused variants
    from cudolfinx.batch import VariantTuner
    from cudolfinx import _lib
    tuner = VariantTuner(reps=1)
    assert tuner.choose(a, A1, None, None) == "atomic"
