"""Forms given as FFCx bodies, without a GPU: the translation units the engine
generates (fe_ffcx_source) compile with NVRTC for sm_100a, and the oracle's
quadrature-evaluated forms -- the reference values of tests/test_gpu_ffcx.py
-- are pinned by exact identities, closed forms and finite differences."""
import ctypes

import numpy as np
import pytest

import ffcx_bodies as fb
from conftest import ensure_library
from oracle import fem_oracle as fo

INTEGRAL = {"cell": 0, "exterior_facet": 1, "interior_facet": 2}

# (builder, test (k, bs), trial (k, bs))
CASES = [
    (lambda: fb.stiffness(1, "dg0"), (4, 1), (4, 1)),
    (lambda: fb.stiffness(2, "p1"), (10, 1), (10, 1)),
    (fb.stiffness_plus_mass, (4, 1), (4, 1)),
    (fb.elasticity, (10, 3), (10, 3)),
    (fb.mixed_p2_p1, (10, 1), (4, 1)),
    (lambda: fb.nonlinear(0), None, None),
    (lambda: fb.nonlinear(1), (4, 1), None),
    (lambda: fb.nonlinear(2), (4, 1), (4, 1)),
    (lambda: fb.robin_mass(1), (4, 1), (4, 1)),
    (lambda: fb.exterior_nonlinear(1), (4, 1), None),
    (lambda: fb.exterior_nonlinear(2), (4, 1), (4, 1)),
    (fb.interior_jump, (4, 1), (4, 1)),
    (fb.interior_sipg, (4, 1), (4, 1)),
    (lambda: fb.interior_nonlinear(0), None, None),
    (lambda: fb.interior_nonlinear(1), (4, 1), None),
    (lambda: fb.interior_nonlinear(2), (4, 1), (4, 1)),
]


def _source(B, test, trial):
    ensure_library()
    from cudolfinx import _lib

    k0, bs0 = test if test else (1, 1)
    k1, bs1 = trial if trial else (1, 1)
    sizes = B["coefficient_sizes"]
    arr = (ctypes.c_int * max(1, len(sizes)))(*sizes)
    n = ctypes.c_int64()
    args = (INTEGRAL[B["integral_type"]], B["rank"], k0, bs0, k1, bs1, len(sizes), arr, B["name"].encode(),
            B["body"].encode())
    _lib.check(_lib.lib.fe_ffcx_source(*args, None, 0, ctypes.byref(n)), "fe_ffcx_source")
    buf = ctypes.create_string_buffer(n.value + 1)
    _lib.check(_lib.lib.fe_ffcx_source(*args, buf, n.value + 1, ctypes.byref(n)), "fe_ffcx_source")
    return buf.value.decode()


def _nvrtc_compile(src):
    L = ctypes.CDLL("libnvrtc.so.12")
    prog = ctypes.c_void_p()
    assert L.nvrtcCreateProgram(ctypes.byref(prog), src.encode(), b"form.cu", 0, None, None) == 0
    opts = [b"-arch=sm_100a", b"-std=c++17"]
    rc = L.nvrtcCompileProgram(prog, len(opts), (ctypes.c_char_p * len(opts))(*opts))
    n = ctypes.c_size_t()
    L.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
    log = ctypes.create_string_buffer(n.value + 1)
    L.nvrtcGetProgramLog(prog, log)
    L.nvrtcDestroyProgram(ctypes.byref(prog))
    return rc, log.value.decode()


@pytest.mark.parametrize("case", range(len(CASES)))
def test_generated_units_compile_for_sm100a(case):
    build, test, trial = CASES[case]
    B = build()
    src = _source(B, test, trial)
    kernels = {0: "fe_ffcx_scalar", 1: "fe_ffcx_vec", 2: "fe_ffcx_mat"}[B["rank"]]
    assert kernels in src and B["name"] in src and B["body"] in src
    rc, log = _nvrtc_compile(src)
    assert rc == 0, log


def test_generated_source_rejects_invalid_names():
    ensure_library()
    from cudolfinx import _lib

    n = ctypes.c_int64()
    st = _lib.lib.fe_ffcx_source(0, 2, 4, 1, 4, 1, 0, None, b"not an identifier", b"", None, 0, ctypes.byref(n))
    assert st == 1 and "identifier" in _lib.last_error()


def test_quadrature_rules_are_exact_to_their_degree():
    for n in (2, 3, 4):
        X, w = fo.tet_rule(n)
        for a in range(2 * n - 2):
            for b in range(2 * n - 2 - a):
                for c in range(2 * n - 2 - a - b):
                    exact = float(fo._mono_int(a, b, c))
                    assert abs(np.sum(w * X[:, 0] ** a * X[:, 1] ** b * X[:, 2] ** c) - exact) < 1e-14
        P, wt = fo.tri_rule(n)
        from math import factorial
        for a in range(2 * n - 1):
            for b in range(2 * n - 1 - a):
                exact = factorial(a) * factorial(b) / factorial(a + b + 2)
                assert abs(np.sum(wt * P[:, 0] ** a * P[:, 1] ** b) - exact) < 1e-14


def test_facet_permutations_match_the_points_of_both_cells():
    coords, cells = fo.unit_cube_tet_mesh(3, jitter=0.2, seed=1)
    perm = np.random.default_rng(0).permutation(len(coords))
    coords, cells = coords[np.argsort(perm)], perm[cells]
    q = fo.interior_facets(cells)
    P2, _ = fo.tri_rule(3)
    codes = set()
    for c0, f0, c1, f1 in q:
        pts = []
        for c, f in ((c0, f0), (c1, f1)):
            code = fo.facet_permutation(cells[c][list(fo.TET_FACETS[f])])
            codes.add(code)
            Xr = fo.facet_points(f, fo.permute_facet_points(P2, code))
            x = coords[cells[c]]
            pts.append(x[0] + Xr @ (x[1:] - x[0]))
        assert np.allclose(pts[0], pts[1], atol=1e-14)
    assert codes == set(range(6))


def test_quadrature_matrices_equal_the_exact_element_tensors():
    coords, cells = fo.unit_cube_tet_mesh(2, jitter=0.2, seed=3)
    K1 = fo.quad_cell_matrix(coords, cells, 1, 1, lambda V0, G0, V1, G1: np.einsum("cqia,cqja->cqij", G0, G1), n=2)
    assert np.allclose(K1, fo.p1_stiffness(coords, cells), rtol=0, atol=1e-14)
    K2 = fo.quad_cell_matrix(coords, cells, 2, 2, lambda V0, G0, V1, G1: np.einsum("cqia,cqja->cqij", G0, G1), n=3)
    assert np.allclose(K2, fo.p2_stiffness(coords, cells, np.ones((len(cells), 4))), rtol=0, atol=1e-13)
    M1 = fo.quad_cell_matrix(coords, cells, 1, 1,
                             lambda V0, G0, V1, G1: np.broadcast_to(V0[None, :, :, None] * V1[None, :, None, :],
                                                                    G0.shape[:2] + (4, 4)), n=3)
    assert np.allclose(M1, fo.mass_matrices(coords, cells, 1), rtol=0, atol=1e-15)


def _fd_check(fun, x0, jac, eps=1e-6):
    """Central differences of fun at x0 against jac (columns = inputs)."""
    cols = []
    for j in range(x0.size):
        e = np.zeros_like(x0)
        e.flat[j] = eps
        cols.append((fun(x0 + e) - fun(x0 - e)) / (2 * eps))
    return np.allclose(np.stack(cols, axis=-1), jac, rtol=1e-6, atol=1e-8)


def test_nonlinear_oracle_forms_are_consistent():
    coords, cells = fo.unit_cube_tet_mesh(2, jitter=0.2, seed=5)
    rng = np.random.default_rng(1)
    u = rng.uniform(-0.5, 0.5, (len(cells), 4))
    kap = rng.uniform(0.5, 2.0, (len(cells), 4))
    R, J, M = fo.quad_cell_forms(coords, cells, u, kap)
    # the Jacobian is the derivative of the residual, cell by cell
    for c in (0, 7, 20):
        f = lambda x: fo.quad_cell_forms(coords, cells[c:c + 1], x[None], kap[c:c + 1])[0][0]
        assert _fd_check(f, u[c].copy(), J[c])
    # u = 0: the residual is the kappa-weighted load, the functional int kappa
    R0, J0, M0 = fo.quad_cell_forms(coords, cells, np.zeros_like(u), kap)
    Mm = fo.mass_matrices(coords, cells, 1)
    assert np.allclose(R0, np.einsum("cij,cj->ci", Mm, kap), atol=1e-14)
    assert np.allclose(M0, Mm.sum(axis=2).__mul__(kap).sum(axis=1), atol=1e-14)
    # exterior: sum_i R_i = int_dOmega u grad u . n = int_Omega |grad u|^2 for linear u, kappa = 1
    F = fo.exterior_facets(cells)
    a = np.array([0.3, -1.2, 0.7])
    ul = (coords @ a)[cells]
    Rf, Jf = fo.exterior_facet_forms(coords, cells, F, ul, np.ones_like(ul))
    assert abs(Rf.sum() - a @ a) < 1e-12
    for e in (0, 5, 30):
        f = lambda x: fo.exterior_facet_forms(coords, cells, F[e:e + 1], np.where(
            np.arange(len(cells))[:, None] == F[e, 0], x[None], ul), kap)[0][0]
        assert _fd_check(f, ul[F[e, 0]].copy(), fo.exterior_facet_forms(coords, cells, F[e:e + 1], ul, kap)[1][0])


def test_interior_oracle_forms_are_consistent():
    coords, cells = fo.unit_cube_tet_mesh(2, jitter=0.2, seed=6)
    q = fo.interior_facets(cells)
    rng = np.random.default_rng(2)
    u = rng.standard_normal((len(cells), 4))
    kv = rng.uniform(0.5, 2.0, len(coords))
    R, J, M, S = fo.interior_facet_forms(coords, cells, q, u, kv, cells, 5.0)
    _, _, _, S0 = fo.interior_facet_forms(coords, cells, q, u, kv, cells, 0.0)
    # the penalty part is 5 x the exact jump tensor
    assert np.allclose((S - S0) / 5.0, fo.interior_jump_tensors(coords, cells, q, 1), rtol=1e-12, atol=1e-15)
    # the consistency terms are symmetric, and vanish on a continuous linear field paired with itself
    assert np.allclose(S0, np.transpose(S0, (0, 2, 1)), atol=1e-14)
    # Jacobian = derivative of the residual in the macro u
    for e in (0, 9):
        c0, c1 = q[e, 0], q[e, 2]

        def f(x):
            uu = u.copy()
            uu[c0], uu[c1] = x[:4], x[4:]
            return fo.interior_facet_forms(coords, cells, q[e:e + 1], uu, kv, cells, 0.0)[0][0]
        assert _fd_check(f, np.concatenate([u[c0], u[c1]]), J[e])
