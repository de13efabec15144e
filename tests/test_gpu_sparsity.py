"""Device-built CSR pattern (fe_sparsity_build_device) against the host
builder, bit for bit: P1, P2, vector P2, rectangular (P2 rows x P1 columns),
a randomly renumbered dofmap and an empty mesh."""
import numpy as np
import pytest

from conftest import ensure_library

from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


def _spaces(n, renumber_seed=None):
    ensure_library()
    from cudolfinx import fem
    mesh = fem.create_unit_cube(n)
    out = {"P1": fem.functionspace(mesh, ("P", 1)), "P2": fem.functionspace(mesh, ("P", 2)),
           "VP2": fem.functionspace(mesh, ("P", 2, (3,)))}
    if renumber_seed is not None:
        rng = np.random.default_rng(renumber_seed)
        V = out["P2"]
        perm = rng.permutation(V.num_nodes).astype(np.int32)
        V.dofs = perm[V.dofs]
    return out


def _compare(V0, V1):
    from cudolfinx.context import get_cuda_context
    from cudolfinx.form import DeviceDofMap
    from cudolfinx.la import Sparsity
    ctx = get_cuda_context()
    d0, d1 = DeviceDofMap(ctx, V0), DeviceDofMap(ctx, V1)
    host = Sparsity.build(ctx, d0, d1, on_device=False)
    dev = Sparsity.build(ctx, d0, d1, on_device=True)
    hr, hc = host.to_host()
    dr, dc = dev.to_host()
    assert np.array_equal(hr, dr) and np.array_equal(hc, dc)
    return dr, dc


@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_device_pattern_matches_host(n):
    S = _spaces(n)
    for name in ("P1", "P2", "VP2"):
        rp, col = _compare(S[name], S[name])
        kind = {"P1": "p1", "P2": "p2", "VP2": "vp2"}[name]
        assert len(col) == fo.nnz_formula(kind, n)
    _compare(S["P2"], S["P1"])   # rectangular
    _compare(S["P1"], S["P2"])


def test_device_pattern_renumbered_dofs():
    S = _spaces(4, renumber_seed=7)
    rp, col = _compare(S["P2"], S["P2"])
    P = fo.build_problem("p2", 4)
    ref_rp, ref_col = fo.sparsity(S["P2"].dofs, S["P2"].dofs, S["P2"].num_nodes)
    assert np.array_equal(rp, ref_rp) and np.array_equal(col, ref_col)
