"""Exterior-facet (ds) forms through the C-ABI against the oracle: Robin mass
(P1, P2) with BCs and accumulated onto a stiffness matrix, Neumann loads (P1,
P2; constant, DG0 and P1 data), vector-P2 traction, and the lifting of a
facet mass form."""
import numpy as np
import pytest

from gpu_util import tolerance_check

from conftest import ensure_library
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


def _setup(deg, n=3):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem
    mesh = fem.create_unit_cube(n)
    V = fem.functionspace(mesh, ("P", deg))
    P = fo.build_problem("p1" if deg == 1 else "p2", n, seed=2)
    assert np.array_equal(V.dofs, P["dofs"])
    return cx, fem, mesh, V, P


@pytest.mark.parametrize("deg", [1, 2])
def test_facet_mass_matches_oracle(deg):
    cx, fem, mesh, V, P = _setup(deg)
    rng = np.random.default_rng(1)
    alpha = rng.uniform(0.5, 2.0, size=mesh.num_cells)
    W = fem.functionspace(mesh, ("DG", 0))
    asm = cx.CUDAAssembler()
    af = cx.form(fem.facet_mass(V, fem.Function(W, alpha)))
    g = fem.Function(V, P["g"])
    bcs = asm.pack_bcs([fem.dirichletbc(g, P["bc_dofs"])])
    # Robin term alone, with BCs
    A = asm.assemble_matrix(af, bcs=bcs)
    A.assemble()
    F = fo.exterior_facets(P["cells"])
    Ae = fo.facet_mass(P["coords"], P["cells"], F, deg, alpha[F[:, 0]])
    rp, col = fo.sparsity(P["dofs"], P["dofs"], P["ndof"])
    mk = np.zeros(P["ndof"], dtype=np.uint8)
    mk[P["bc_dofs"]] = 1
    fd = P["dofs"][F[:, 0]]
    ref = fo.assemble_matrix(Ae, fd, fd, rp, col, bc0_markers=mk, bc1_markers=mk, bc0_owned_dofs=P["bc_dofs"])
    bound = fo.matrix_bound(Ae, fd, fd, rp, col, bc0_markers=mk, bc1_markers=mk)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref, bound)
    assert ok, worst
    # stiffness + Robin: the second call accumulates (zero=False)
    k = 1.0
    a = cx.form(fem.stiffness(V, k))
    A2 = asm.assemble_matrix(a, bcs=bcs)
    asm.assemble_matrix(af, A2, bcs=bcs, zero=False)
    A2.assemble()
    Ks = fo.p1_stiffness(P["coords"], P["cells"]) if deg == 1 else \
        fo.p2_stiffness(P["coords"], P["cells"], np.ones((len(P["cells"]), 4)))
    ref2 = fo.assemble_matrix(Ks, P["dofs"], P["dofs"], rp, col, bc0_markers=mk, bc1_markers=mk,
                              bc0_owned_dofs=P["bc_dofs"])
    ref2 += ref
    diag = fo.diag_positions(rp, col)[P["bc_dofs"]]
    ref2[diag] = 1.0   # set_diagonal sets the value again, it does not add
    bound2 = bound + fo.matrix_bound(Ks, P["dofs"], P["dofs"], rp, col, bc0_markers=mk, bc1_markers=mk)
    ok, worst = tolerance_check(A2.values.cpu().numpy(), ref2, bound2)
    assert ok, worst


@pytest.mark.parametrize("deg", [1, 2])
@pytest.mark.parametrize("gkind", ["constant", "dg0", "p1"])
def test_facet_load_matches_oracle(deg, gkind):
    cx, fem, mesh, V, P = _setup(deg)
    rng = np.random.default_rng(3)
    if gkind == "constant":
        g, gspec = 2.5, 2.5
    elif gkind == "dg0":
        g = rng.uniform(-1, 1, size=mesh.num_cells)
        gspec = fem.Function(fem.functionspace(mesh, ("DG", 0)), g)
    else:
        g = rng.uniform(-1, 1, size=len(P["coords"]))
        gspec = fem.Function(fem.functionspace(mesh, ("P", 1)), g)
    asm = cx.CUDAAssembler()
    L = cx.form(fem.facet_load(V, gspec))
    b = asm.assemble_vector(L).to_host()
    F = fo.exterior_facets(P["cells"])
    be = fo.facet_load(P["coords"], P["cells"], F, deg, g, gkind, p1_cells=P["cells"])
    ref = fo.assemble_vector(be, P["dofs"][F[:, 0]], P["ndof"])
    ok, worst = tolerance_check(b, ref, fo.vector_bound(be, P["dofs"][F[:, 0]], P["ndof"]))
    assert ok, worst


def test_vector_traction_matches_oracle():
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem
    P = fo.build_problem("vp2", 2, seed=1)
    mesh = fem.Mesh(P["coords"], P["cells"], grid_n=2)
    V = fem.functionspace(mesh, ("P", 2, (3,)))
    asm = cx.CUDAAssembler()
    t = (0.5, -1.0, 2.0)
    b = asm.assemble_vector(cx.form(fem.facet_load(V, np.array(t)))).to_host()
    F = fo.exterior_facets(P["cells"])
    be = fo.facet_vector_load(P["coords"], P["cells"], F, t)
    ref = fo.assemble_vector(be, P["dofs"][F[:, 0]], 3 * P["ndof"], bs=3)
    ok, worst = tolerance_check(b, ref, fo.vector_bound(be, P["dofs"][F[:, 0]], 3 * P["ndof"], bs=3))
    assert ok, worst


@pytest.mark.parametrize("deg", [1, 2])
def test_facet_mass_lifting(deg):
    cx, fem, mesh, V, P = _setup(deg)
    asm = cx.CUDAAssembler()
    af = cx.form(fem.facet_mass(V, 1.5))
    g = fem.Function(V, P["g"])
    bcs = asm.pack_bcs([fem.dirichletbc(g, P["bc_dofs"][::2])])  # every other boundary dof
    L = cx.form(fem.load(V, 1.0))
    b = asm.assemble_vector(L)
    b0 = b.to_host().copy()
    asm.apply_lifting(b, [af], [bcs], scale=0.75)
    F = fo.exterior_facets(P["cells"])
    Ae = fo.facet_mass(P["coords"], P["cells"], F, deg, 1.5)
    mk = np.zeros(P["ndof"], dtype=np.uint8)
    mk[P["bc_dofs"][::2]] = 1
    fd = P["dofs"][F[:, 0]]
    ref = fo.apply_lifting(b0.copy(), Ae, fd, fd, mk, P["g"], scale=0.75)
    # b0 (the engine's load vector) is the common start of both sums
    bound = fo.lifting_bound(P["ndof"], Ae, fd, fd, mk, P["g"], scale=0.75) + fo.PARITY_RTOL * np.abs(b0)
    ok, worst = tolerance_check(b.to_host(), ref, bound)
    assert ok, worst


def test_facet_form_errors():
    cx, fem, mesh, V, P = _setup(1, n=2)
    asm = cx.CUDAAssembler()
    af = cx.form(fem.facet_mass(V, 1.0))
    with pytest.raises(RuntimeError, match="atomic scatter only"):
        asm.assemble_matrix(af, variant="deterministic")
    from cudolfinx import _lib
    bad = np.array([[0, 4]], dtype=np.int32)
    with pytest.raises(RuntimeError, match="local facet"):
        _lib.check(_lib.lib.fe_form_set_facets(af.cuda_form, bad.ctypes.data, 1), "fe_form_set_facets")
