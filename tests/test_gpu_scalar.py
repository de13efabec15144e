"""Functionals (fe_assemble_scalar) against the oracle and known answers:
int f dx (constant, DG0, P1), int k |grad u|^2 dx for P1 / P2 u (= u^T A u),
int g ds over exterior facets; repeated calls give the same bits."""
import numpy as np
import pytest

from conftest import ensure_library
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _env(n=3):
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem
    return cx, fem, fem.create_unit_cube(n)


def test_integral_constant_dg0_p1():
    cx, fem, mesh = _env()
    asm = cx.CUDAAssembler()
    assert abs(asm.assemble_scalar(cx.form(fem.integral(2.0, mesh))) - 2.0) < RTOL
    coords, cells = fo.unit_cube_tet_mesh(3)
    _, det, _ = fo.cell_geometry(coords, cells)
    vol = np.abs(det) / 6.0
    rng = np.random.default_rng(0)
    f0 = rng.uniform(-1, 1, size=mesh.num_cells)
    W = fem.functionspace(mesh, ("DG", 0))
    v = asm.assemble_scalar(cx.form(fem.integral(fem.Function(W, f0))))
    assert abs(v - np.dot(vol, f0)) < RTOL * np.abs(vol * f0).sum()
    V1 = fem.functionspace(mesh, ("P", 1))
    f1 = rng.uniform(-1, 1, size=V1.num_dofs)
    v = asm.assemble_scalar(cx.form(fem.integral(fem.Function(V1, f1))))
    ref = np.dot(vol, f1[cells].mean(axis=1))
    assert abs(v - ref) < RTOL * np.abs(vol[:, None] * f1[cells]).sum()


@pytest.mark.parametrize("deg", [1, 2])
def test_energy_equals_uAu(deg):
    cx, fem, mesh = _env()
    asm = cx.CUDAAssembler()
    V = fem.functionspace(mesh, ("P", deg))
    W = fem.functionspace(mesh, ("DG", 0))
    rng = np.random.default_rng(deg)
    k = np.exp(rng.standard_normal(mesh.num_cells))
    u = rng.uniform(-1, 1, size=V.num_dofs)
    kf = fem.Function(W, k)
    e = asm.assemble_scalar(cx.form(fem.energy(fem.Function(V, u), kf)))
    coords, cells = fo.unit_cube_tet_mesh(3)
    Ae = fo.p1_stiffness(coords, cells, k) if deg == 1 else fo.p2_stiffness(coords, cells, np.repeat(k[:, None], 4, 1))
    ue = u[V.dofs]
    ref = np.einsum("ci,cij,cj->", ue, Ae, ue)
    assert abs(e - ref) < 1e-11 * abs(ref)
    # the same value from the assembled stiffness matrix (no BCs)
    A = asm.assemble_matrix(cx.form(fem.stiffness(V, kf))).mat
    assert abs(e - u @ (A @ u)) < 1e-11 * abs(ref)


def test_facet_integral():
    cx, fem, mesh = _env()
    asm = cx.CUDAAssembler()
    assert abs(asm.assemble_scalar(cx.form(fem.facet_integral(1.0, mesh))) - 6.0) < 1e-12
    V1 = fem.functionspace(mesh, ("P", 1))
    g = V1.tabulate_dof_coordinates().sum(axis=1)
    assert abs(asm.assemble_scalar(cx.form(fem.facet_integral(fem.Function(V1, g), mesh))) - 9.0) < 1e-12


def test_scalar_bitwise_repeatable():
    cx, fem, mesh = _env(6)
    asm = cx.CUDAAssembler()
    V = fem.functionspace(mesh, ("P", 2))
    u = np.random.default_rng(5).standard_normal(V.num_dofs)
    M = cx.form(fem.energy(fem.Function(V, u), 1.5))
    vals = {asm.assemble_scalar(M) for _ in range(4)}
    assert len(vals) == 1
