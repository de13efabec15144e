"""CPU tests of the product's host side: the C-ABI library loads and exports
every declared entry point, the host pattern builder is bit-exact with the
oracle (DOLFINx SparsityPattern + la/petsc.cpp:45-65 unroll), and the
cudolfinx.fem stand-ins generate the oracle's meshes and dofmaps."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, ensure_library
from oracle import fem_oracle as fo

HEADER = os.path.join(ROOT, "include", "cudolfinx_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fe_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    path = ensure_library()
    lib = ctypes.CDLL(path)
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_declares_every_symbol():
    ensure_library()
    from cudolfinx import _lib

    assert set(declared_symbols()) == set(_lib.EXPORTED)


def _host_pattern(d0, d1, bs, nb):
    from cudolfinx import _lib

    nnz = ctypes.c_int64()
    rp, cl = ctypes.c_void_p(), ctypes.c_void_p()
    d0 = np.ascontiguousarray(d0, dtype=np.int32)
    d1 = np.ascontiguousarray(d1, dtype=np.int32)
    st = _lib.lib.fe_pattern_build_host(d0.ctypes.data, d1.ctypes.data, d0.shape[0], d0.shape[1], d1.shape[1], bs, bs,
                                        nb, nb, ctypes.byref(nnz), ctypes.byref(rp), ctypes.byref(cl))
    if st != 0:
        return st, _lib.last_error(), None
    nrows = nb * bs
    row_ptr = np.ctypeslib.as_array((ctypes.c_int32 * (nrows + 1)).from_address(rp.value)).copy()
    col = np.ctypeslib.as_array((ctypes.c_int32 * max(1, nnz.value)).from_address(cl.value))[: nnz.value].copy()
    _lib.lib.fe_free_host(rp)
    _lib.lib.fe_free_host(cl)
    return st, row_ptr, col


@pytest.mark.parametrize("kind,n", [("p1", 1), ("p1", 4), ("p2", 1), ("p2", 3), ("vp2", 2)])
def test_host_pattern_bit_exact_with_oracle(kind, n):
    ensure_library()
    P = fo.build_problem(kind, n)
    st, rp, col = _host_pattern(P["dofs"], P["dofs"], P["bs"], P["ndof"])
    assert st == 0, rp
    ref_rp, ref_col = fo.sparsity(P["dofs"], P["dofs"], P["ndof"], P["bs"], P["bs"])
    assert np.array_equal(rp, ref_rp)
    assert np.array_equal(col, ref_col)


def test_host_pattern_rectangular_and_ragged():
    # rows from a P1 map, columns from a P2 map on the same cells (rectangular, uneven rows)
    ensure_library()
    P1 = fo.build_problem("p1", 2)
    dofs2, nd2, _ = fo.p2_dofmap(2, P1["cells"])
    from cudolfinx import _lib

    nnz = ctypes.c_int64()
    rp, cl = ctypes.c_void_p(), ctypes.c_void_p()
    d0 = np.ascontiguousarray(P1["dofs"], dtype=np.int32)
    d1 = np.ascontiguousarray(dofs2, dtype=np.int32)
    st = _lib.lib.fe_pattern_build_host(d0.ctypes.data, d1.ctypes.data, len(d0), 4, 10, 1, 1, P1["ndof"], nd2,
                                        ctypes.byref(nnz), ctypes.byref(rp), ctypes.byref(cl))
    assert st == 0
    n0 = P1["ndof"]
    row_ptr = np.ctypeslib.as_array((ctypes.c_int32 * (n0 + 1)).from_address(rp.value)).copy()
    col = np.ctypeslib.as_array((ctypes.c_int32 * nnz.value).from_address(cl.value)).copy()
    _lib.lib.fe_free_host(rp)
    _lib.lib.fe_free_host(cl)
    ref_rp, ref_col = fo.sparsity(P1["dofs"], dofs2, n0)
    assert np.array_equal(row_ptr, ref_rp) and np.array_equal(col, ref_col)


def test_host_pattern_empty_mesh():
    ensure_library()
    st, rp, col = _host_pattern(np.zeros((0, 4), np.int32), np.zeros((0, 4), np.int32), 1, 5)
    assert st == 0 and np.array_equal(rp, np.zeros(6, np.int32)) and len(col) == 0


def test_host_pattern_rejects_out_of_range_dofs():
    ensure_library()
    d = np.array([[0, 1, 2, 7]], dtype=np.int32)
    st, msg, _ = _host_pattern(d, d, 1, 4)
    assert st == 1 and "out of range" in msg


@pytest.mark.parametrize("n,jitter", [(2, 0.0), (3, 0.2)])
def test_fem_standins_match_oracle(n, jitter):
    ensure_library()
    from cudolfinx import fem

    m = fem.create_unit_cube(n, jitter=jitter, seed=0)
    coords, cells = fo.unit_cube_tet_mesh(n, jitter=jitter, seed=0)
    assert np.array_equal(m.cells, cells) and np.array_equal(m.geometry_x, coords)
    V2 = fem.functionspace(m, ("P", 2))
    dofs, nd, grid = fo.p2_dofmap(n, cells)
    assert V2.num_nodes == nd and np.array_equal(V2.dofs, dofs)
    assert np.array_equal(V2.boundary_nodes(), fo.boundary_dofs_from_grid(grid, 2 * n))
    X = fo.dof_coordinates(coords, cells, dofs, nd, 2)
    assert np.allclose(V2.tabulate_dof_coordinates(), X)
    V1 = fem.functionspace(m, ("P", 1))
    assert np.array_equal(V1.boundary_nodes(), fo.boundary_dofs_from_grid(fo.vertex_grid_index(n), n))
    Vv = fem.functionspace(m, ("P", 2, (3,)))
    assert Vv.bs == 3 and Vv.num_dofs == 3 * nd
    V3 = fem.functionspace(m, ("P", 3))
    d3, nd3, grid3 = fo.p3_dofmap(n, cells)
    assert V3.num_nodes == nd3 and np.array_equal(V3.dofs, d3)
    assert np.array_equal(V3.boundary_nodes(), fo.boundary_dofs_from_grid(grid3, 3 * n))
    assert np.allclose(V3.tabulate_dof_coordinates(), fo.dof_coordinates(coords, cells, d3, nd3, 3))


def test_p3_form_specs_build_without_gpu():
    from cudolfinx import fem
    mesh = fem.create_unit_cube(2)
    V3 = fem.functionspace(mesh, ("P", 3))
    assert fem.stiffness(V3, 2.0).kind == "P3_STIFFNESS"
    assert fem.stiffness(V3, 2.0, precision="fp32").precision == "fp32"
    assert fem.load(V3, 1.0).kind == "P3_LOAD"
    for bad in (lambda: fem.facet_mass(V3), lambda: fem.facet_load(V3, 1.0),
                lambda: fem.energy(fem.Function(V3)), lambda: fem.functionspace(mesh, ("P", 3, (3,))),
                lambda: fem.functionspace(mesh, ("P", 4))):
        with pytest.raises(ValueError):
            bad()


def test_functional_specs_build_without_gpu():
    from cudolfinx import fem
    mesh = fem.create_unit_cube(2)
    V2 = fem.functionspace(mesh, ("P", 2))
    u = fem.Function(V2, np.ones(V2.num_dofs))
    s = fem.energy(u, 2.0)
    assert s.rank == 0 and s.kind == "P2_ENERGY" and s.mesh is mesh and s.function_spaces == []
    assert fem.integral(1.0, mesh).kind == "INTEGRAL"
    fi = fem.facet_integral(1.0, mesh)
    assert fi.kind == "FACET_INTEGRAL" and len(fi.facets) == 12 * 4
    with pytest.raises(ValueError):
        fem.energy(fem.Function(fem.functionspace(mesh, ("P", 2, (3,)))))


def test_reference_nodes_and_basis_are_lagrange_and_match_the_oracle():
    from cudolfinx import fem
    m = fem.create_unit_cube(1)
    spaces = {0: fem.functionspace(m, ("DG", 0)), 1: fem.functionspace(m, ("P", 1)),
              2: fem.functionspace(m, ("P", 2)), 3: fem.functionspace(m, ("P", 3))}
    for d, V in spaces.items():
        X = fem.reference_nodes(V)
        assert np.allclose(X, fo.element_nodes(d))
        if d:
            assert np.allclose(fem.lagrange_basis(V, X), np.eye(len(X)), atol=1e-14)
    for dt in spaces:
        for ds in (1, 2, 3):
            assert np.allclose(fem.interpolation_matrix(spaces[dt], spaces[ds]), fo.interpolation_operator(dt, ds),
                               atol=1e-14)


def test_mass_specs_and_form_part_validation_without_gpu():
    import cudolfinx as cx
    from cudolfinx import fem
    from cudolfinx import _lib
    mesh = fem.create_unit_cube(2)
    V1, V2 = fem.functionspace(mesh, ("P", 1)), fem.functionspace(mesh, ("P", 2))
    V2v = fem.functionspace(mesh, ("P", 2, (3,)))
    for V, kind in ((V1, "P1_MASS"), (V2, "P2_MASS"), (V2v, "VP2_MASS")):
        s = fem.mass(V, 2.0)
        assert s.kind == kind and s.rank == 2 and s.precision == "fp64" and kind in _lib.FORM
    for bad in (lambda: fem.mass(fem.functionspace(mesh, ("P", 3))),
                lambda: fem.mass(fem.functionspace(mesh, ("DG", 1)))):
        with pytest.raises(ValueError):
            bad()
    # the "part" option is checked before any device work
    opts = {"form_compiler_options": {"part": "diagonal"}}
    with pytest.raises(ValueError, match="one space"):
        cx.form(fem.load(V2, 1.0), **opts)
    with pytest.raises(ValueError, match="one space"):
        cx.form(fem.facet_mass(V1, 1.0, fem.exterior_facets(mesh)), **opts)
    with pytest.raises(ValueError, match="unknown form part"):
        cx.form(fem.stiffness(V2, 1.0), form_compiler_options={"part": "lower"})


def test_variant_tuner_key_separates_coefficient_kinds():
    from cudolfinx import fem
    from cudolfinx.batch import VariantTuner
    mesh = fem.create_unit_cube(2)
    V1 = fem.functionspace(mesh, ("P", 1))
    W = fem.functionspace(mesh, ("DG", 0))

    class _Form:  # the tuner keys on the form spec only
        def __init__(self, spec):
            self._spec = spec

    keys = {VariantTuner.key(_Form(fem.stiffness(V1, k)))
            for k in (1.0, fem.Function(W, np.ones(mesh.num_cells)), fem.Function(V1, np.ones(V1.num_dofs)))}
    assert len(keys) == 3


def test_interior_facets_and_dg_specs_without_gpu():
    from cudolfinx import fem
    mesh = fem.create_unit_cube(3, jitter=0.1, seed=2)
    q = fem.interior_facets(mesh)
    ext = fem.exterior_facets(mesh)
    C = mesh.num_cells
    assert 2 * len(q) + len(ext) == 4 * C                      # every facet once, interior ones twice
    assert np.all(q[:, 0] < q[:, 2]) and q[:, [1, 3]].min() >= 0 and q[:, [1, 3]].max() <= 3
    tri = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])
    v0 = np.sort(mesh.cells[q[:, 0][:, None], tri[q[:, 1]]], axis=1)
    v1 = np.sort(mesh.cells[q[:, 2][:, None], tri[q[:, 3]]], axis=1)
    assert np.array_equal(v0, v1)                               # the two sides name the same facet
    ref = fo.interior_facets(mesh.cells)
    assert sorted(map(tuple, q.tolist())) == sorted(map(tuple, np.asarray(ref).tolist()))
    V0, V1 = fem.functionspace(mesh, ("DG", 0)), fem.functionspace(mesh, ("DG", 1))
    assert fem.jump_penalty(V0, 2.0).kind == "DG0_JUMP" and fem.jump_penalty(V1).kind == "DG1_JUMP"
    assert np.array_equal(fem.jump_penalty(V1).facets, q)
    L = fem.facet_average_load(V1, 1.0, q[:5])
    assert L.kind == "DG1_AVG_LOAD" and L.rank == 1 and len(L.facets) == 5
    Vp = fem.functionspace(mesh, ("P", 1))
    assert fem.jump_norm(fem.Function(Vp)).kind == "JUMP_NORM"
    for bad in (lambda: fem.jump_norm(fem.Function(fem.functionspace(mesh, ("P", 2)))),
                lambda: fem.jump_norm(fem.Function(fem.functionspace(mesh, ("P", 2, (3,)))))):
        with pytest.raises(ValueError):
            bad()


def test_boundary_dofs_bcs_and_elasticity_specs_without_gpu():
    from cudolfinx import fem
    mesh = fem.create_unit_cube(2)
    V = fem.functionspace(mesh, ("P", 2))
    Vv = fem.functionspace(mesh, ("P", 2, (3,)))
    s = fem.locate_boundary_dofs(V)
    v = fem.locate_boundary_dofs(Vv)
    assert np.array_equal(v, (s[:, None] * 3 + np.arange(3)).ravel())
    X = V.tabulate_dof_coordinates()
    on = np.any((X < 1e-12) | (X > 1 - 1e-12), axis=1)
    assert np.array_equal(np.sort(s), np.nonzero(on)[0])
    bc = fem.dirichletbc(0.5, s, V)
    bcv = fem.dirichletbc(fem.Function(Vv, np.ones(Vv.num_dofs)), v)
    assert bc is not None and bcv is not None
    assert fem.elasticity(Vv, 1.0, 2.0).kind == "VP2_ELASTICITY"
    with pytest.raises(ValueError):
        fem.elasticity(V, 1.0, 2.0)


def test_fused_rhs_validates_its_arguments_on_the_host():
    ensure_library()
    from cudolfinx import _lib

    st = _lib.lib.fe_assemble_rhs(None, None, None, None, None, 1.0, 0, None)
    assert st != 0 and "null form" in _lib.last_error()


def test_assembly_graph_branches_balance_nonzeros_and_keep_forms_together():
    # the capture's split of the items over parallel branches: each form's
    # items on one branch, largest forms first onto the least-loaded branch
    from types import SimpleNamespace

    ensure_library()
    from cudolfinx.batch import AssemblyGraph

    forms = [object() for _ in range(6)]
    sizes = [900, 500, 400, 300, 200, 100]
    g = object.__new__(AssemblyGraph)
    g.items = [{"a": f, "mat": SimpleNamespace(sparsity=SimpleNamespace(nnz=n))} for f, n in zip(forms, sizes)]
    g.items.append({"a": forms[0], "mat": SimpleNamespace(sparsity=SimpleNamespace(nnz=50))})  # a second item of form 0
    groups = g._branch_items(3)
    assert sorted(len(x) for x in groups) == [2, 2, 3]
    flat = [it for grp in groups for it in grp]
    assert len(flat) == len(g.items) and all(any(it is x for x in flat) for it in g.items)
    for grp in groups:  # both items of form 0 share a branch
        if any(it["a"] is forms[0] for it in grp):
            assert sum(it["a"] is forms[0] for it in grp) == 2
    loads = sorted(sum(it["mat"].sparsity.nnz for it in grp) for grp in groups)
    assert loads == [700, 800, 950]
    assert len(g._branch_items(1)) == 1
    assert len(g._branch_items(16)) == 6  # no empty branches
