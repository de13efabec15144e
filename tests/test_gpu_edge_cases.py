"""Edge cases of the block, restricted, interior-facet and interpolation
paths: empty facet lists and restrictions, mismatched spaces, and the errors
they must raise (no GPU fault, the context stays usable)."""
import numpy as np
import pytest

from conftest import ensure_library
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


def _cx():
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem
    return cx, fem


def test_interior_facet_forms_with_no_facets():
    cx, fem = _cx()
    mesh = fem.create_unit_cube(2)
    V = fem.functionspace(mesh, ("DG", 1))
    none = np.zeros((0, 4), dtype=np.int32)
    asm = cx.CUDAAssembler()
    A = asm.assemble_matrix(cx.form(fem.jump_penalty(V, 1.0, facets=none)))
    A.assemble()
    assert A.sparsity.nnz == 0
    b = asm.assemble_vector(cx.form(fem.facet_average_load(V, 1.0, facets=none)))
    assert np.all(b.to_host() == 0.0)
    u = fem.Function(V, np.arange(V.num_dofs, dtype=np.float64))
    assert asm.assemble_scalar(cx.form(fem.jump_norm(u, facets=none))) == 0.0


def test_block_system_with_an_empty_restriction():
    cx, fem = _cx()
    mesh = fem.create_unit_cube(2)
    V = fem.functionspace(mesh, ("P", 1))
    W = fem.functionspace(mesh, ("P", 1))
    empty = np.zeros(0, dtype=np.int32)
    a = cx.form([[fem.stiffness(V), fem.stiffness(V, trial=W)], [fem.stiffness(W, trial=V), fem.stiffness(W)]],
                restriction=([None, empty], [None, empty]))
    assert a.row_offsets == [0, V.num_dofs, V.num_dofs]
    asm = cx.CUDAAssembler()
    M = asm.assemble_matrix_block(a)
    M.assemble()
    ref = asm.assemble_matrix(cx.form(fem.stiffness(V)))
    ref.assemble()
    rp, col = M.sparsity.to_host()
    rp0, col0 = ref.sparsity.to_host()
    assert np.array_equal(rp, rp0) and np.array_equal(col, col0)
    P = fo.build_problem("p1", 2, seed=0)
    Ae = fo.p1_stiffness(P["coords"], P["cells"])
    ok, worst = fo.within_bound(M.values.cpu().numpy(), fo.assemble_matrix(Ae, V.dofs, V.dofs, rp0, col0),
                                fo.matrix_bound(Ae, V.dofs, V.dofs, rp0, col0))
    assert ok, worst


def test_union_pattern_rejects_forms_on_other_spaces():
    cx, fem = _cx()
    mesh = fem.create_unit_cube(2)
    V1 = fem.functionspace(mesh, ("DG", 1))
    V0 = fem.functionspace(mesh, ("DG", 0))
    asm = cx.CUDAAssembler()
    with pytest.raises(RuntimeError, match="other sizes"):
        asm.create_matrix([cx.form(fem.jump_penalty(V1)), cx.form(fem.jump_penalty(V0))])
    # the context stays usable
    A = asm.assemble_matrix(cx.form(fem.jump_penalty(V0)))
    A.assemble()
    assert A.sparsity.nnz > 0


def test_interpolation_rejects_other_meshes_and_block_sizes():
    cx, fem = _cx()
    m1, m2 = fem.create_unit_cube(2), fem.create_unit_cube(3)
    c1 = cx.Coefficient(fem.Function(fem.functionspace(m1, ("P", 2))))
    c2 = cx.Coefficient(fem.Function(fem.functionspace(m2, ("P", 1))))
    with pytest.raises(ValueError, match="different meshes"):
        c1.interpolate(c2)
    cv = cx.Coefficient(fem.Function(fem.functionspace(m1, ("P", 2, (3,)))))
    with pytest.raises(RuntimeError, match="block size"):
        cv.interpolate(cx.Coefficient(fem.Function(fem.functionspace(m1, ("P", 1)))))
