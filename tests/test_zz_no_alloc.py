"""GPU test of fe_pcg_solve_noalloc, the allocation-free Jacobi-PCG entry point.

Who needs it: callers that cannot allocate device memory while they solve.
An application that has already given the card's memory to its own pool (a
framework caching allocator, or a PETSc / Kokkos arena sized to the device)
may see cudaMalloc fail or take memory from that budget, and a latency-bound
loop must not enter the CUDA allocator, which can synchronise the device.
The entry point keeps its scratch vectors in one static device array instead.

The test calls it through the C-ABI on two different systems in a row (the
second call reuses the scratch left by the first) and compares each result
with the allocating fe_pcg_solve: both run the same kernels with the same
launch shapes, so the iterates agree bitwise on one GPU.  Around a call it
also checks the property itself: the device's free memory (cudaMemGetInfo)
and torch's allocator counters do not move.  It also checks the size limit.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from gpu_util import run_system
from oracle import fem_oracle as fo

pytestmark = pytest.mark.gpu

NOALLOC_MAX_ROWS = 1 << 18


def _solve(fn, A, b, x, rtol, max_iter, stream):
    it, res = ctypes.c_int(0), ctypes.c_double(0.0)
    st = fn(A.sparsity.handle, A.values.data_ptr(), b.vector.data_ptr(), x.data_ptr(), rtol, max_iter,
            ctypes.byref(it), ctypes.byref(res), stream)
    return st, it.value, res.value


def _alloc_state(torch):
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    st = torch.cuda.memory_stats()
    return free, st.get("allocation.all.allocated", 0), torch.cuda.memory_reserved()


def test_noalloc_pcg_matches_allocating_solver_on_two_calls_in_a_row():
    import torch

    from cudolfinx import _lib

    for kind, n, seed in (("p2", 6, 11), ("p1", 9, 12)):
        P = fo.build_problem(kind, n, seed=seed)
        R = run_system(P)
        A, b = R["Aobj"], R["bobj"]
        stream = torch.cuda.current_stream().cuda_stream
        x_ref = torch.zeros(b.size, dtype=torch.float64, device="cuda")
        x_na = torch.zeros(b.size, dtype=torch.float64, device="cuda")
        x_na2 = torch.zeros(b.size, dtype=torch.float64, device="cuda")
        st_ref, it_ref, res_ref = _solve(_lib.lib.fe_pcg_solve, A, b, x_ref, 1e-10, 5000, stream)
        st_na, it_na, res_na = _solve(_lib.lib.fe_pcg_solve_noalloc, A, b, x_na, 1e-10, 5000, stream)
        assert st_ref == 0, _lib.last_error()
        assert st_na == 0, _lib.last_error()
        # a call made after one call on this device (which loaded the module
        # holding the static scratch) changes neither the device's free memory
        # nor torch's allocator
        before = _alloc_state(torch)
        st_na2, it_na2, res_na2 = _solve(_lib.lib.fe_pcg_solve_noalloc, A, b, x_na2, 1e-10, 5000, stream)
        after = _alloc_state(torch)
        assert st_na2 == 0, _lib.last_error()
        assert after == before, f"device memory moved across the call: {before} -> {after}"
        assert it_na == it_ref == it_na2 and it_na > 0
        assert res_na <= 1e-10 and res_na == res_ref == res_na2
        x_ref_h, x_na_h = x_ref.cpu().numpy(), x_na.cpu().numpy()
        assert np.array_equal(x_na_h, x_ref_h), f"{kind} n={n}: results differ from fe_pcg_solve"
        assert np.array_equal(x_na2.cpu().numpy(), x_ref_h)


def test_noalloc_pcg_rejects_matrices_above_its_limit():
    import torch

    import cudolfinx as cx
    from cudolfinx import _lib

    n = NOALLOC_MAX_ROWS + 1
    ctx = cx.get_cuda_context()
    rp = np.arange(n + 1, dtype=np.int32)
    col = np.arange(n, dtype=np.int32)
    S = cx.Sparsity.from_csr(ctx, rp, col, n)
    vals = torch.ones(n, dtype=torch.float64, device="cuda")
    b = torch.ones(n, dtype=torch.float64, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    it, res = ctypes.c_int(0), ctypes.c_double(0.0)
    st = _lib.lib.fe_pcg_solve_noalloc(S.handle, vals.data_ptr(), b.data_ptr(), x.data_ptr(), 1e-8, 10,
                                       ctypes.byref(it), ctypes.byref(res), torch.cuda.current_stream().cuda_stream)
    assert st == 1
    assert str(NOALLOC_MAX_ROWS) in _lib.last_error()
