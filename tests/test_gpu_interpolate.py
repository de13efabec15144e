"""Device interpolation (cudolfinx.Coefficient.interpolate -> fe_interpolate)
against the oracle's restatement of the reference algorithm
(interpolate_same_map: gather, multiply by the interpolation operator, scatter).

Continuous sources give the same value at a shared target dof from every
cell, so the engine's owner-cell choice and the reference's last-writer
choice agree to rounding: tolerance 1e-13 relative to max|u|.  Interpolating
a polynomial of the source degree is exact.
"""
import numpy as np
import pytest

from conftest import ensure_library
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu

SPACES = {"DG0": ("DG", 0), "P1": ("P", 1), "P2": ("P", 2), "P3": ("P", 3)}
DEG = {"DG0": 0, "P1": 1, "P2": 2, "P3": 3}


@pytest.mark.parametrize("src,dst", [("P1", "P2"), ("P1", "P3"), ("P2", "P3"), ("P3", "P2"), ("P2", "P1"),
                                     ("P3", "P1"), ("P1", "DG0"), ("P2", "DG0"), ("P2", "P2")])
def test_interpolation_matches_oracle(src, dst):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    n = 4
    mesh = fem.create_unit_cube(n, jitter=0.2, seed=2)
    V0 = fem.functionspace(mesh, SPACES[src])
    V1 = fem.functionspace(mesh, SPACES[dst])
    rng = np.random.default_rng(5)
    u0 = fem.Function(V0, rng.standard_normal(V0.num_dofs))
    c0 = cx.Coefficient(u0)
    c1 = cx.Coefficient(fem.Function(V1))
    c1.interpolate(c0)
    ref = fo.interpolate_same_map(u0.x.array, V0.dofs, V1.dofs, fo.interpolation_operator(DEG[dst], DEG[src]),
                                  V1.num_dofs)
    got = c1.values()
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    assert np.array_equal(got, c1.device_values.cpu().numpy())


def test_interpolation_is_exact_for_polynomials_and_vector_spaces():
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    mesh = fem.create_unit_cube(5, jitter=0.15, seed=1)
    V2 = fem.functionspace(mesh, ("P", 2))
    V3 = fem.functionspace(mesh, ("P", 3))
    q = lambda X: 1 + X[:, 0] - 2 * X[:, 1] * X[:, 2] + X[:, 2] ** 2
    u2 = fem.Function(V2, q(V2.tabulate_dof_coordinates()))
    c3 = cx.Coefficient(fem.Function(V3))
    c3.interpolate(cx.Coefficient(u2))
    assert np.abs(c3.values() - q(V3.tabulate_dof_coordinates())).max() < 1e-13
    # vector P2 -> vector P2 (component by component) is the identity
    W = fem.functionspace(mesh, ("P", 2, (3,)))
    w = fem.Function(W, np.random.default_rng(0).standard_normal(W.num_dofs))
    cw = cx.Coefficient(fem.Function(W))
    cw.interpolate(cx.Coefficient(w))
    assert np.abs(cw.values() - w.x.array).max() < 1e-14
