"""Equispaced P3 on the GPU: the element-free identities at sizes the oracle
does not reach, and the P3 error paths.

A cubic u is interpolated exactly by P3, so with k = 1 and no BCs
u^T A u = int |grad u|^2 and sum_i b_i u_i = int u (f = 1) over the unit cube,
on any affine mesh of it; both sides are known in closed form (tensor Gauss
rule).  Relative tolerance 1e-11 (FP64 element tensors, FP64 atomics).
"""
import numpy as np
import pytest

from conftest import ensure_library

pytestmark = pytest.mark.gpu


def _cube_gauss(fun, q=4):
    t, w = np.polynomial.legendre.leggauss(q)
    t, w = 0.5 * (t + 1.0), 0.5 * w
    Z, Y, X = np.meshgrid(t, t, t, indexing="ij")
    W = (w[:, None, None] * w[None, :, None] * w[None, None, :]).ravel()
    return float(np.sum(W * fun(X.ravel(), Y.ravel(), Z.ravel())))


def _u(x, y, z):
    return x ** 3 + y ** 2 * z + x * y * z - 2.0 * z ** 3


def _grad2(x, y, z):
    gx = 3 * x ** 2 + y * z
    gy = 2 * y * z + x * z
    gz = y ** 2 + x * y - 6 * z ** 2
    return gx * gx + gy * gy + gz * gz


@pytest.mark.parametrize("n,jitter,variant", [(6, 0.2, "atomic"), (20, 0.15, "atomic"),
                                              (6, 0.2, "deterministic"), (20, 0.15, "auto")])
def test_p3_cubic_energy_and_load_identities(n, jitter, variant):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem
    import scipy.sparse as sp

    mesh = fem.create_unit_cube(n, jitter=jitter, seed=n)
    V = fem.functionspace(mesh, ("P", 3))
    X = V.tabulate_dof_coordinates()
    u = _u(X[:, 0], X[:, 1], X[:, 2])
    asm = cx.CUDAAssembler()
    a = cx.form(fem.stiffness(V, 1.0))
    L = cx.form(fem.load(V, 1.0))
    A = asm.assemble_matrix(a, variant=variant)
    A.assemble()
    b = asm.assemble_vector(L).to_host()
    rp, col = A.sparsity.to_host()
    N = V.num_dofs
    assert rp[-1] == 1311 * n ** 3 + 459 * n ** 2 + 45 * n + 1
    M = sp.csr_matrix((A.values.cpu().numpy(), col, rp), shape=(N, N))
    e = float(u @ (M @ u))
    ref = _cube_gauss(_grad2)
    assert abs(e - ref) <= 1e-11 * ref
    assert abs(float(b @ u) - _cube_gauss(_u)) <= 1e-12
    assert abs(b.sum() - 1.0) <= 1e-12
    # constants are in the kernel of the assembled operator
    assert np.abs(M @ np.ones(N)).max() <= 1e-11 * np.abs(M.data).max()


def test_p3_rejects_unsupported_variants_and_coefficients():
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    mesh = fem.create_unit_cube(2)
    V = fem.functionspace(mesh, ("P", 3))
    asm = cx.CUDAAssembler()
    a = cx.form(fem.stiffness(V, 1.0))
    for variant in ("tile", "block", "row-gather"):
        with pytest.raises(RuntimeError):
            asm.assemble_matrix(a, variant=variant)
    V1 = fem.functionspace(mesh, ("P", 1))
    with pytest.raises(RuntimeError, match="P1 coefficients"):
        cx.form(fem.stiffness(V, fem.Function(V1, np.ones(V1.num_dofs))))
