"""Request server on the GPU: each result is the same alone and in the mix,
FP32-element results stay within 1e-6 of the FP64 path, a P1 request matches
the oracle, and admission keeps the device-memory ledger within its budget."""
import numpy as np
import pytest

from conftest import ensure_library

from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu

# alone vs in the mix with the default (FP64-atomic) assembly: the matrices
# differ in summation order only, and both PCG runs stop at rtol 1e-8, so the
# solutions agree to the stated solution tolerance
MIX_TOL = 1e-6
FP32_TOL = 1e-6     # FP32 element tensors vs the FP64 path (relative 2-norm of the solution)


def _requests(count=10, seed=4, nmin=3, nmax=6):
    ensure_library()
    from cudolfinx import serve
    return serve.make_requests(count, rate=0.0, seed=seed, nmin=nmin, nmax=nmax)


def test_alone_equals_mixed():
    variant = "auto"
    from cudolfinx import serve
    reqs = _requests()
    alone = []
    srv1 = serve.Server(workers=1, precision="fp32", variant=variant)
    for r in reqs:
        alone += srv1.run([r])
    srv4 = serve.Server(workers=4, precision="fp32", variant=variant)
    mixed = srv4.run(reqs)
    assert srv4.max_concurrent > 1
    for a, m in zip(alone, mixed):
        assert a.error is None and m.error is None, (a.error, m.error)
        assert a.rel_residual <= 1e-8 and m.rel_residual <= 1e-8
        assert serve.solution_difference(m, a) < MIX_TOL, (m.kind, m.n)


def test_fp32_server_within_tolerance_of_plain_fp64():
    from cudolfinx import serve
    reqs = _requests(count=9, seed=7)
    for r in reqs:
        r.rtol = 1e-12  # compare the discretisations, not where two PCG runs stop
    plain = serve.Server(plain=True).run(reqs)
    fast = serve.Server(workers=3, precision="fp32").run(reqs)
    worst = 0.0
    for p, f in zip(plain, fast):
        assert p.error is None and f.error is None
        worst = max(worst, serve.solution_difference(f, p))
    assert worst < FP32_TOL, worst


def test_p1_request_matches_oracle():
    import scipy.sparse.linalg as spla
    from cudolfinx import serve
    req = [r for r in _requests(count=30, seed=11) if r.kind == "p1"][0]
    res = serve.Server(workers=1, precision="fp64").run([req])[0]
    n = req.n
    coords, cells = fo.unit_cube_tet_mesh(n)
    dofs = cells
    N = len(coords)
    grid = fo.vertex_grid_index(n)
    bnd = fo.boundary_dofs_from_grid(grid, n)
    rp, col = fo.sparsity(dofs, dofs, N)
    mk = np.zeros(N, dtype=np.uint8)
    mk[bnd] = 1
    Ae = fo.p1_stiffness(coords, cells, req.coef[0])
    A = fo.assemble_matrix(Ae, dofs, dofs, rp, col, bc0_markers=mk, bc1_markers=mk, bc0_owned_dofs=bnd)
    g = coords.sum(axis=1)
    be = fo.p1_load_p1f(coords, cells, np.ones(N))
    b = fo.assemble_vector(be, dofs, N)
    b = fo.apply_lifting(b, Ae, dofs, dofs, mk, g)
    b = fo.set_bc(b, bnd, g)
    import scipy.sparse as sp
    x = spla.spsolve(sp.csr_matrix((A, col, rp), shape=(N, N)).tocsc(), b)
    err = np.linalg.norm(res.x - x) / np.linalg.norm(x)
    assert err < 1e-6, err


def test_admission_budget_and_oversize_request():
    from cudolfinx import serve
    reqs = _requests(count=8, seed=5, nmin=3, nmax=5)
    C = 6 * 12 ** 3
    big = serve.Request(len(reqs), "vp2", 12, (np.ones(C), np.ones(C)))
    budget = max(serve.slot_bytes(*r.key) + serve.shared_bytes(*r.key) for r in reqs) * 3
    assert serve.slot_bytes(*big.key) + serve.shared_bytes(*big.key) > budget
    srv = serve.Server(workers=4, hbm_budget=budget, precision="fp32")
    out = srv.run(reqs + [big])
    assert all(r.error is None for r in out[:-1])
    assert out[-1].error and "budget" in out[-1].error
    assert srv.ledger.peak <= budget
