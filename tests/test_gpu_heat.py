"""Backward-Euler heat equation through the public API: mass + stiffness into
one matrix, M u^n + dt F from load forms (a P1 load with a P1 coefficient is
M u^n exactly), lifting, set_bc and the on-device PCG, for three steps,
against a direct solve of the oracle's matrices (solution within 1e-8
relative to max|u|: PCG rtol 1e-12 on a well-conditioned M + dt K).
"""
import numpy as np
import pytest

from conftest import ensure_library
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,dt", [(6, 0.05), (10, 0.01)])
def test_backward_euler_steps_match_a_direct_solve(n, dt):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    P = fo.build_problem("p1", n, seed=1)
    mesh = fem.Mesh(P["coords"], P["cells"], grid_n=n)
    V = fem.functionspace(mesh, ("P", 1))
    N = V.num_dofs
    u0 = np.sin(np.pi * P["coords"][:, 0]) * P["coords"][:, 1] * (1 - P["coords"][:, 1])
    un = fem.Function(V, u0)
    asm = cx.CUDAAssembler()
    m = cx.form(fem.mass(V))
    k = cx.form(fem.stiffness(V, dt))
    Lu = cx.form(fem.load(V, un))       # M u^n
    Lf = cx.form(fem.load(V, dt))       # dt * F with f = 1
    bc = fem.dirichletbc(fem.Function(V, np.zeros(N)), P["bc_dofs"])
    bcs = asm.pack_bcs([bc])
    A = asm.assemble_matrix(m, bcs=bcs)
    asm.assemble_matrix(k, A, bcs=bcs, zero=False)
    A.assemble()

    # oracle: A = M + dt K with BC rows/columns removed and a unit diagonal
    dofs = P["dofs"]
    rp, col = fo.sparsity(dofs, dofs, N)
    markers = np.zeros(N, dtype=np.uint8)
    markers[P["bc_dofs"]] = 1
    Me = fo.mass_matrices(P["coords"], P["cells"], 1)
    Ke = fo.p1_stiffness(P["coords"], P["cells"]) * dt
    Aref = fo.assemble_matrix(Me + Ke, dofs, dofs, rp, col, 1, 1, markers, markers, 1.0, P["bc_dofs"])
    Mfull = sp.csr_matrix((fo.assemble_matrix(Me, dofs, dofs, rp, col), col, rp), shape=(N, N))
    Fvec = fo.assemble_vector(fo.p1_load_p1f(P["coords"], P["cells"], np.full(N, dt)), dofs, N)
    As = sp.csr_matrix((Aref, col, rp), shape=(N, N)).tocsc()

    x = None
    uref = u0.copy()
    for step in range(3):
        b = asm.assemble_vector(Lu)
        asm.assemble_vector(Lf, b, zero=False)
        asm.apply_lifting(b, [m], [bcs])
        asm.set_bc(b, bcs, V)
        x, it, res = asm.solve(A, b, x, rtol=1e-12)
        u = x.to_host()
        rhs = Mfull @ uref + Fvec
        rhs[P["bc_dofs"]] = 0.0
        uref = spla.spsolve(As, rhs)
        assert np.abs(u - uref).max() <= 1e-8 * np.abs(uref).max(), (step, it, res)
        un.x.array[:] = u   # next step's M u^n: the load form re-uploads its coefficient
    assert np.abs(u[P["bc_dofs"]]).max() == 0.0
