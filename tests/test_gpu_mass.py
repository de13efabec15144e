"""Cell mass matrices c*inner(u, v)*dx (FE_FORM_P1_MASS / P2_MASS / VP2_MASS) on the GPU.

Checked against the oracle (exact reference mass tensors): values with BC
rows/columns skipped and a unit diagonal, within the oracle's per-entry bound
(fem_oracle.matrix_bound; FP64 atomics add in another order), for constant, DG0
and P1 coefficients and the atomic, full-scatter and deterministic variants;
lifting and the diagonal part; M + dt*K assembled into one matrix; and the
L2 identity u^T M u = int u^2 for u in the space (relative 1e-12).
"""
import numpy as np
import pytest

from conftest import ensure_library
from gpu_util import tolerance_check
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


def _setup(degree, n, coef, seed=0):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    P = fo.build_problem("p1" if degree == 1 else "p2", n, seed=seed)
    mesh = fem.Mesh(P["coords"], P["cells"], grid_n=n)
    V = fem.functionspace(mesh, ("P", degree))
    assert np.array_equal(V.dofs, P["dofs"])
    rng = np.random.default_rng(seed + 17)
    C = len(P["cells"])
    if coef == "const":
        c, kw = 2.5, dict(c_dg0=np.full(C, 2.5))
    elif coef == "dg0":
        vals = rng.uniform(0.5, 3.0, C)
        c, kw = fem.Function(fem.functionspace(mesh, ("DG", 0)), vals), dict(c_dg0=vals)
    else:
        vals = rng.uniform(0.5, 3.0, len(P["coords"]))
        c, kw = fem.Function(fem.functionspace(mesh, ("P", 1)), vals), dict(c_vertex=vals[P["cells"]])
    Ae = fo.mass_matrices(P["coords"], P["cells"], degree, **kw)
    return cx, fem, P, mesh, V, c, Ae


@pytest.mark.parametrize("degree,n", [(1, 6), (2, 4)])
@pytest.mark.parametrize("coef", ["const", "dg0", "p1"])
@pytest.mark.parametrize("variant", ["auto", "atomic-full", "deterministic"])
def test_mass_matrix_with_bcs_matches_oracle(degree, n, coef, variant):
    cx, fem, P, mesh, V, c, Ae = _setup(degree, n, coef, seed=n)
    asm = cx.CUDAAssembler()
    a = cx.form(fem.mass(V, c))
    bc = fem.dirichletbc(fem.Function(V, P["g"]), P["bc_dofs"])
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


@pytest.mark.parametrize("degree,n", [(1, 5), (2, 4)])
def test_mass_lifting_diagonal_and_time_step_matrix(degree, n):
    cx, fem, P, mesh, V, c, Ae = _setup(degree, n, "p1", seed=3)
    asm = cx.CUDAAssembler()
    m = cx.form(fem.mass(V, c))
    bc = fem.dirichletbc(fem.Function(V, P["g"]), P["bc_dofs"])
    bcs = asm.pack_bcs([bc])
    markers = np.zeros(P["ndof"], dtype=np.uint8)
    markers[P["bc_dofs"]] = 1
    # lifting: b = 0 - M (g on the BC columns)
    L = cx.form(fem.load(V, 0.0))
    b = asm.assemble_vector(L)
    asm.apply_lifting(b, [m], [bcs])
    ref_b = fo.apply_lifting(np.zeros(P["ndof"]), Ae, P["dofs"], P["dofs"], markers, P["g"])
    bound_b = fo.lifting_bound(P["ndof"], Ae, P["dofs"], P["dofs"], markers, P["g"])
    ok, worst = tolerance_check(b.to_host(), ref_b, bound_b)
    assert ok, worst
    # diagonal part: the lumping / Jacobi vector of M
    d = asm.assemble_vector(cx.form(fem.mass(V, c), form_compiler_options={"part": "diagonal"})).to_host()
    ok, worst = tolerance_check(d, fo.assemble_diagonal(Ae, P["dofs"], P["ndof"]),
                                fo.diagonal_bound(Ae, P["dofs"], P["ndof"]))
    assert ok, worst
    # M + dt K in one matrix: stiffness added onto the mass values (same pattern)
    dt = 0.05
    k = cx.form(fem.stiffness(V, dt))
    A = asm.assemble_matrix(m)
    asm.assemble_matrix(k, A, zero=False)
    A.assemble()
    rp, col = A.sparsity.to_host()
    if degree == 1:
        Ke = fo.p1_stiffness(P["coords"], P["cells"]) * dt
    else:
        Ke = fo.p2_stiffness(P["coords"], P["cells"], np.full((len(P["cells"]), 4), dt))
    ref = fo.assemble_matrix(Ae + Ke, P["dofs"], P["dofs"], rp, col)
    # two assemblies into one matrix: the contributions of both
    bound = fo.matrix_bound(Ae, P["dofs"], P["dofs"], rp, col) + fo.matrix_bound(Ke, P["dofs"], P["dofs"], rp, col)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref, bound)
    assert ok, worst


@pytest.mark.parametrize("degree", [1, 2])
def test_mass_reproduces_l2_norm_of_a_polynomial_in_the_space(degree):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem
    import scipy.sparse as sp

    mesh = fem.create_unit_cube(6, jitter=0.2, seed=2)
    V = fem.functionspace(mesh, ("P", degree))
    X = V.tabulate_dof_coordinates()
    x, y, z = X[:, 0], X[:, 1], X[:, 2]
    if degree == 1:
        u = 1.0 + x - 2.0 * y + 3.0 * z
        exact = 1 + 14 / 3 + 2 + 2 * (-2 + 3 - 6) / 4
    else:
        u = x * x - y * z + x
        # int (x^2 + x - yz)^2 = int x^4 + x^2 + y^2 z^2 + 2x^3 - 2x^2 yz - 2x yz
        exact = 1 / 5 + 1 / 3 + 1 / 9 + 2 / 4 - 2 * (1 / 3) * (1 / 4) - 2 * (1 / 2) * (1 / 4)
    A = cx.CUDAAssembler().assemble_matrix(cx.form(fem.mass(V)))
    A.assemble()
    rp, col = A.sparsity.to_host()
    M = sp.csr_matrix((A.values.cpu().numpy(), col, rp), shape=(V.num_dofs, V.num_dofs))
    assert abs(u @ (M @ u) - exact) <= 1e-12 * exact
    assert abs(M.sum() - 1.0) <= 1e-13  # the volume of the unit cube


def test_mass_rejects_the_stiffness_only_variants():
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    mesh = fem.create_unit_cube(2)
    asm = cx.CUDAAssembler()
    for degree in (1, 2):
        a = cx.form(fem.mass(fem.functionspace(mesh, ("P", degree))))
        for variant in ("tile", "block"):
            with pytest.raises(RuntimeError):
                asm.assemble_matrix(a, variant=variant)
    with pytest.raises(ValueError):
        fem.mass(fem.functionspace(mesh, ("P", 3)))


@pytest.mark.parametrize("coef", ["const", "dg0", "p1"])
@pytest.mark.parametrize("variant", ["auto", "atomic-full", "deterministic"])
def test_vector_p2_mass_matches_oracle(coef, variant):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    n = 3
    P = fo.build_problem("vp2", n, seed=5)
    mesh = fem.Mesh(P["coords"], P["cells"], grid_n=n)
    V = fem.functionspace(mesh, ("P", 2, (3,)))
    rng = np.random.default_rng(8)
    C = len(P["cells"])
    if coef == "const":
        c, kw = 1.7, dict(c_dg0=np.full(C, 1.7))
    elif coef == "dg0":
        vals = rng.uniform(0.5, 3.0, C)
        c, kw = fem.Function(fem.functionspace(mesh, ("DG", 0)), vals), dict(c_dg0=vals)
    else:
        vals = rng.uniform(0.5, 3.0, len(P["coords"]))
        c, kw = fem.Function(fem.functionspace(mesh, ("P", 1)), vals), dict(c_vertex=vals[P["cells"]])
    Ae = fo.vector_mass(fo.mass_matrices(P["coords"], P["cells"], 2, **kw))
    asm = cx.CUDAAssembler()
    m = cx.form(fem.mass(V, c))
    bc = fem.dirichletbc(fem.Function(V, np.linspace(-1.0, 1.0, 3 * P["ndof"])), P["bc_dofs"])
    bcs = asm.pack_bcs([bc])
    A = asm.assemble_matrix(m, bcs=bcs, variant=variant)
    A.assemble()
    rp, col = A.sparsity.to_host()
    nscal = 3 * P["ndof"]
    markers = np.zeros(nscal, dtype=np.uint8)
    markers[P["bc_dofs"]] = 1
    ref = fo.assemble_matrix(Ae, P["dofs"], P["dofs"], rp, col, 3, 3, markers, markers, 1.0, P["bc_dofs"])
    bound = fo.matrix_bound(Ae, P["dofs"], P["dofs"], rp, col, 3, 3, markers, markers)
    ok, worst = tolerance_check(A.values.cpu().numpy(), ref, bound)
    assert ok, worst
    if variant == "auto":
        L0 = cx.form(fem.load(V, np.zeros(3)))
        b = asm.assemble_vector(L0)
        asm.apply_lifting(b, [m], [bcs])
        g = np.linspace(-1.0, 1.0, nscal)
        ok, worst = tolerance_check(b.to_host(), fo.apply_lifting(np.zeros(nscal), Ae, P["dofs"], P["dofs"],
                                                                  markers, g, bs0=3, bs1=3),
                                    fo.lifting_bound(nscal, Ae, P["dofs"], P["dofs"], markers, g, bs0=3, bs1=3))
        assert ok, worst
        d = asm.assemble_vector(cx.form(fem.mass(V, c), form_compiler_options={"part": "diagonal"})).to_host()
        ok, worst = tolerance_check(d, fo.assemble_diagonal(Ae, P["dofs"], nscal, 3),
                                    fo.diagonal_bound(Ae, P["dofs"], nscal, 3))
        assert ok, worst


def test_vector_p2_mass_reproduces_the_l2_norm_of_a_quadratic_field():
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem
    import scipy.sparse as sp

    mesh = fem.create_unit_cube(5, jitter=0.2, seed=6)
    V = fem.functionspace(mesh, ("P", 2, (3,)))
    X = V.tabulate_dof_coordinates()
    x, y, z = X[:, 0], X[:, 1], X[:, 2]
    u = np.stack([x * x, y * z, np.ones_like(x)], axis=1).ravel()  # (x^2, yz, 1)
    exact = 1 / 5 + 1 / 9 + 1.0
    A = cx.CUDAAssembler().assemble_matrix(cx.form(fem.mass(V, 2.0)))
    A.assemble()
    rp, col = A.sparsity.to_host()
    M = sp.csr_matrix((A.values.cpu().numpy(), col, rp), shape=(u.size, u.size))
    assert abs(u @ (M @ u) - 2.0 * exact) <= 1e-12 * exact
