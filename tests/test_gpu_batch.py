"""Batched assembly of many DG0-coefficient instances on one mesh and pattern
(fe_assemble_matrix_batch) against the oracle, per instance.

Element tensors are FP32 by design, so the bound is the FP32 one: relative
Frobenius error below 1e-6 and every entry within 1e-6 of the largest entry
of its matrix."""
import numpy as np
import pytest

from gpu_util import mirror_problem

from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu

FROB_TOL = 1e-6
ENTRY_TOL = 1e-6


def _instances(P, S, seed):
    rng = np.random.default_rng(seed)
    C = len(P["cells"])
    return [np.exp(rng.uniform(np.log(1e-2), np.log(1e2), size=C)) for _ in range(S)]


def _oracle_matrix(P, k, diagonal=1.0, with_bc=True):
    dofs = P["dofs"]
    rp, col = fo.sparsity(dofs, dofs, P["ndof"])
    if P["degree"] == 1:
        Ae = fo.p1_stiffness(P["coords"], P["cells"], k)
    else:
        Ae = fo.p2_stiffness(P["coords"], P["cells"], np.repeat(k[:, None], 4, axis=1))
    markers = None
    if with_bc:
        markers = np.zeros(P["ndof"], dtype=np.uint8)
        markers[P["bc_dofs"]] = 1
    A = fo.assemble_matrix(Ae, dofs, dofs, rp, col, bc0_markers=markers, bc1_markers=markers, diagonal=diagonal,
                           bc0_owned_dofs=P["bc_dofs"] if with_bc else None)
    return rp, col, A


def _check(gpu, ref):
    frob = np.linalg.norm(gpu - ref) / np.linalg.norm(ref)
    worst = np.abs(gpu - ref).max() / np.abs(ref).max()
    assert frob < FROB_TOL, f"relative Frobenius error {frob:.3e}"
    assert worst < ENTRY_TOL, f"max entry error {worst:.3e} of max|A|"


def _setup(kind, n):
    import torch
    P = fo.build_problem("p1k" if kind == "p1" else "p2", n, seed=3)
    M = mirror_problem(P)
    cx = M["cx"]
    from cudolfinx import fem
    W = fem.functionspace(M["mesh"], ("DG", 0))
    a = cx.form(fem.stiffness(M["V"], fem.Function(W, np.ones(len(P["cells"])))))
    asm = cx.CUDAAssembler()
    bcs = asm.pack_bcs([M["bc"]])
    return P, M, a, asm, bcs, torch


@pytest.mark.parametrize("kind,n,S", [("p1", 4, 5), ("p1", 6, 40), ("p2", 3, 7), ("p2", 4, 33), ("p2", 3, 70)])
def test_batch_matches_oracle(kind, n, S):
    P, M, a, asm, bcs, torch = _setup(kind, n)
    ks = _instances(P, S, seed=11)
    kd = [torch.tensor(k, device="cuda") for k in ks]
    mats = asm.assemble_matrix_batch(a, kd, bcs=bcs)
    torch.cuda.synchronize()
    for k, m in zip(ks, mats):
        rp, col, ref = _oracle_matrix(P, k)
        hrp, hcol = m.sparsity.to_host()
        assert np.array_equal(hrp, rp) and np.array_equal(hcol, col)
        _check(m.values.cpu().numpy(), ref)


def test_batch_bitwise_reproducible_and_matches_single():
    P, M, a, asm, bcs, torch = _setup("p1", 5)
    ks = _instances(P, 70, seed=5)
    kd = torch.tensor(np.stack(ks), device="cuda")
    m1 = asm.assemble_matrix_batch(a, kd, bcs=bcs)
    v1 = [m.values.clone() for m in m1]
    m2 = asm.assemble_matrix_batch(a, kd, mats=m1, bcs=bcs)
    torch.cuda.synchronize()
    for x, m in zip(v1, m2):
        assert torch.equal(x, m.values)
    # instance 17 through the single-instance FP64 path with the same k
    from cudolfinx import fem
    W = fem.functionspace(M["mesh"], ("DG", 0))
    a17 = M["cx"].form(fem.stiffness(M["V"], fem.Function(W, ks[17])))
    A17 = asm.assemble_matrix(a17, bcs=bcs)
    A17.assemble()
    _check(m2[17].values.cpu().numpy(), A17.values.cpu().numpy())


def test_batch_accumulate_no_bc_and_diagonal():
    P, M, a, asm, bcs, torch = _setup("p1", 4)
    ks = _instances(P, 3, seed=9)
    kd = [torch.tensor(k, device="cuda") for k in ks]
    # without BCs
    mats = asm.assemble_matrix_batch(a, kd)
    torch.cuda.synchronize()
    for k, m in zip(ks, mats):
        _, _, ref = _oracle_matrix(P, k, with_bc=False)
        _check(m.values.cpu().numpy(), ref)
    # zero=False accumulates; BC rows keep their old values, BC diagonal is set
    for m in mats:
        m.values.fill_(1.0)
    mats = asm.assemble_matrix_batch(a, kd, mats=mats, bcs=bcs, diagonal=2.5, zero=False)
    torch.cuda.synchronize()
    for k, m in zip(ks, mats):
        rp, col, ref = _oracle_matrix(P, k, diagonal=2.5)
        expect = 1.0 + ref
        rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
        bcd = np.zeros(P["ndof"], dtype=bool)
        bcd[P["bc_dofs"]] = True
        expect[bcd[rows] & (rows == col)] = 2.5
        _check(m.values.cpu().numpy(), expect)


def test_batch_more_instances_than_one_launch():
    P, M, a, asm, bcs, torch = _setup("p1", 2)
    ks = _instances(P, 450, seed=2)
    kd = torch.tensor(np.stack(ks), device="cuda")
    mats = asm.assemble_matrix_batch(a, kd, bcs=bcs)
    torch.cuda.synchronize()
    for i in (0, 63, 64, 127, 128, 383, 384, 449):
        _, _, ref = _oracle_matrix(P, ks[i])
        _check(mats[i].values.cpu().numpy(), ref)


def test_batch_empty_and_unsupported():
    P, M, a, asm, bcs, torch = _setup("p1", 2)
    assert asm.assemble_matrix_batch(a, []) == []
    Pv = fo.build_problem("vp2", 2, seed=1)
    Mv = mirror_problem(Pv)
    av = Mv["cx"].form(Mv["a"])
    kd = [torch.ones(len(Pv["cells"]), dtype=torch.float64, device="cuda")]
    with pytest.raises(RuntimeError, match="P1/P2 stiffness"):
        asm.assemble_matrix_batch(av, kd)


def test_batch_second_call_with_new_coefficients():
    # two calls into the same matrices with different coefficients: the
    # second must see only its own packed coefficients (nothing of the first
    # call's packed copy may be read back through a cache)
    P, M, a, asm, bcs, torch = _setup("p1", 5)
    k1 = _instances(P, 40, seed=21)
    k2 = _instances(P, 40, seed=22)
    mats = asm.assemble_matrix_batch(a, torch.tensor(np.stack(k1), device="cuda"), bcs=bcs)
    mats = asm.assemble_matrix_batch(a, torch.tensor(np.stack(k2), device="cuda"), mats=mats, bcs=bcs)
    torch.cuda.synchronize()
    for i in (0, 17, 39):
        rp, col, ref = _oracle_matrix(P, k2[i])
        _check(mats[i].values.cpu().numpy(), ref)
