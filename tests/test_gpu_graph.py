"""Many meshes of different sizes, P1, P2 and P3 mixed, assembled by one CUDA
graph replay (cudolfinx.AssemblyGraph) against the oracle; the variant
autotuner's choice per item is one of the parity-tested variants."""
import numpy as np
import pytest

from gpu_util import mirror_problem, tolerance_check

from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu

CASES = [("p1", 3, "fp64"), ("p2", 2, "fp32"), ("p1", 5, "fp64"), ("p2", 3, "fp64"), ("p1k", 4, "fp64"),
         ("p2", 4, "fp32"), ("p3", 2, "fp64"), ("p3", 3, "fp32")]


def _items():
    import torch  # noqa: F401
    out = []
    for kind, n, prec in CASES:
        P = fo.build_problem(kind, n, seed=n)
        M = mirror_problem(P, precision=prec)
        cx = M["cx"]
        asm = cx.CUDAAssembler()
        a = cx.form(M["a"])
        mat = asm.create_matrix(a)
        bcs = asm.pack_bcs([M["bc"]])
        ref = fo.solve_system(P)
        out.append((P, prec, a, mat, bcs, ref))
    return out


def _check(mat, ref, prec):
    got = mat.values.cpu().numpy()
    if prec == "fp64":
        ok, worst = tolerance_check(got, ref["A"], ref["A_bound"])
        assert ok, worst
    else:
        frob = np.linalg.norm(got - ref["A"]) / np.linalg.norm(ref["A"])
        assert frob < 2e-6, frob


@pytest.mark.parametrize("variants", ["tune", "auto", "atomic"])
def test_graph_replay_matches_oracle(variants):
    import torch
    import cudolfinx as cx
    its = _items()
    g = cx.AssemblyGraph([(a, mat, bcs) for _, _, a, mat, bcs, _ in its], variants=variants).capture()
    for _, _, _, mat, _, _ in its:
        mat.values.fill_(float("nan"))
    g.replay()
    torch.cuda.synchronize()
    for (P, prec, a, mat, bcs, ref) in its:
        _check(mat, ref, prec)
    # a second replay gives the same matrices again
    for _, _, _, mat, _, _ in its:
        mat.values.fill_(-1.0)
    g.replay()
    torch.cuda.synchronize()
    for (P, prec, a, mat, bcs, ref) in its:
        _check(mat, ref, prec)
    if variants == "tune":
        for it in g.items:
            assert it["variant"] in cx.batch.CANDIDATES[it["a"]._spec.kind]
        assert g.tuner.timings


def test_graph_requires_capture():
    import cudolfinx as cx
    its = _items()[:1]
    g = cx.AssemblyGraph([(a, mat, bcs) for _, _, a, mat, bcs, _ in its], variants="auto")
    with pytest.raises(RuntimeError, match="capture"):
        g.replay()
