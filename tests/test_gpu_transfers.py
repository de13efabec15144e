"""Overlapped transfers: coefficient uploads run on the upload stream after
the last kernels that read the same buffer, read-backs on the download stream
before the next write into the vector.  Assembling several steps in a row
with coefficients that change every step, reading each right-hand side back
asynchronously, must give the same results as running every step to
completion before the next: both within the oracle's per-entry bound of the
oracle's system for that step's coefficients (FP64 atomics sum in any order).
"""
import numpy as np
import pytest
import torch

from gpu_util import mirror_problem, tolerance_check
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu


def _steps(P, overlapped, nsteps=4, rhs_stream=False):
    M = mirror_problem(P)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    a, L = cx.form(M["a"]), cx.form(M["L"])
    k = M["a"].coefficients[0]
    f = M["L"].coefficients[0]
    k0, f0 = k.x.array.copy(), f.x.array.copy()
    A = asm.create_matrix(a)
    b = asm.create_vector(L)
    bcs = asm.pack_bcs([M["bc"]])
    outs, mats = [], []
    side = torch.cuda.Stream() if rhs_stream else None
    for s in range(nsteps):
        k.x.array = k0 * (1.0 + 0.5 * s)
        f.x.array = f0 * (1.0 - 0.25 * s)
        if side is not None:
            side.wait_stream(torch.cuda.current_stream())
        asm.assemble_matrix(a, A, bcs=bcs)
        with torch.cuda.stream(side if side is not None else torch.cuda.current_stream()):
            asm.assemble_vector(L, b)
            asm.apply_lifting(b, [a], [bcs])
            asm.set_bc(b, bcs, M["V"])
            if overlapped:
                outs.append(b.copy_to_host())
        if side is not None:
            torch.cuda.current_stream().wait_stream(side)
        if overlapped:
            mats.append(A.values.clone())
        else:
            torch.cuda.synchronize()
            outs.append(b.to_host().copy())
            mats.append(A.values.clone())
            torch.cuda.synchronize()
    torch.cuda.synchronize()
    return [o.numpy() if hasattr(o, "numpy") else o for o in outs], [m.cpu().numpy() for m in mats]


# p1k n=28: a DG0 k of 131,712 values (1.05 MB), large enough for the upload
# stream and the device copies that uploads rotate through; more steps than
# copies, with the right-hand side on a second stream as well
@pytest.mark.parametrize("kind,n,rhs_stream", [("p2", 5, False), ("p1k", 10, False), ("p1k", 28, False),
                                               ("p1k", 28, True)])
def test_overlapped_transfers_match_synchronous_steps(kind, n, rhs_stream):
    P = fo.build_problem(kind, n, seed=12)
    b_ovl, A_ovl = _steps(P, True, nsteps=5 if n >= 28 else 4, rhs_stream=rhs_stream)
    b_syn, A_syn = _steps(P, False, nsteps=len(b_ovl))
    for s in range(len(b_syn)):
        Ps = dict(P)
        Ps["k"] = P["k"] * (1.0 + 0.5 * s)
        Ps["f"] = P["f"] * (1.0 - 0.25 * s)
        S = fo.solve_system(Ps)
        for b, A in ((b_ovl[s], A_ovl[s]), (b_syn[s], A_syn[s])):
            ok, worst = tolerance_check(b, S["b"], S["b_bound"])
            assert ok, (s, worst)
            ok, worst = tolerance_check(A, S["A"], S["A_bound"])
            assert ok, (s, worst)
    # the steps differ (the coefficients changed), so a stale upload would show
    assert np.abs(b_syn[0] - b_syn[1]).max() > 0
