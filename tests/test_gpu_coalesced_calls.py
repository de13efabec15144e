"""Repeated and graph-replayed calls of the default P2 / vector-P2 matrix
path (warp-coalesced scatter after the zero pass that also stores the BC
diagonal), against the oracle's per-entry bound:
- every slot is written: the values start as NaN before each call;
- repeated calls into the same values, and CUDA-graph replays of one
  captured call;
- zero=False accumulates (no zeroing).
"""
import numpy as np
import pytest

from gpu_util import mirror_problem, tolerance_check
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu

CASES = [("p2", 9), ("vp2", 4), ("vp2", 6)]


def _setup(kind, n, precision="fp64"):
    P = fo.build_problem(kind, n, seed=n + 3)
    M = mirror_problem(P, precision)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    a = cx.form(M["a"])
    bcs = asm.pack_bcs([M["bc"]])
    return P, M, cx, asm, a, bcs


@pytest.mark.parametrize("kind,n", CASES)
def test_every_slot_written_on_repeated_calls(kind, n):
    P, M, cx, asm, a, bcs = _setup(kind, n)
    S = fo.solve_system(P)
    A = asm.create_matrix(a)
    for _ in range(3):
        A.values.fill_(float("nan"))
        asm.assemble_matrix(a, A, bcs=bcs)
        A.assemble()
        vals = A.values.cpu().numpy()
        assert np.isfinite(vals).all()
        ok, worst = tolerance_check(vals, S["A"], S["A_bound"])
        assert ok, worst


@pytest.mark.parametrize("kind,n", CASES)
def test_replayed_in_a_cuda_graph(kind, n):
    import torch

    from cudolfinx import _lib

    P, M, cx, asm, a, bcs = _setup(kind, n)
    S = fo.solve_system(P)
    A = asm.create_matrix(a)
    asm.assemble_matrix(a, A, bcs=bcs)  # plans and BC lists are built outside the capture
    A.assemble()
    h = a.cuda_form
    bc0 = bcs._get_cpp_bcs(a.function_spaces[0], a.restriction(0))
    bc1 = bcs._get_cpp_bcs(a.function_spaces[1], a.restriction(1))
    graph = torch.cuda.CUDAGraph()
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.graph(graph, stream=stream):
        _lib.check(_lib.lib.fe_assemble_matrix(h, A.values.data_ptr(), bc0.handle, bc1.handle, 1.0, _lib.ASM_ZERO,
                                               torch.cuda.current_stream().cuda_stream), "fe_assemble_matrix")
    torch.cuda.synchronize()
    for _ in range(3):
        A.values.fill_(float("nan"))
        graph.replay()
        A.assemble()
        vals = A.values.cpu().numpy()
        assert np.isfinite(vals).all()
        ok, worst = tolerance_check(vals, S["A"], S["A_bound"])
        assert ok, worst
    del graph


@pytest.mark.parametrize("kind,n", CASES)
def test_zero_false_accumulates(kind, n):
    P, M, cx, asm, a, bcs = _setup(kind, n)
    A = asm.assemble_matrix(a)
    A.assemble()
    v1 = A.values.cpu().numpy().copy()
    asm.assemble_matrix(a, A, zero=False)
    A.assemble()
    v2 = A.values.cpu().numpy()
    assert np.abs(v2 - 2.0 * v1).max() <= 1e-13 * np.abs(v1).max()
