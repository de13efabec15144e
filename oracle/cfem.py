"""ctypes driver for the C restatement in cfem.c (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use
this.  The shared library is compiled with ``-O3 -march=native`` for the CPU
it runs on (gcc is present on every box of this image); the file name carries
a fingerprint of the host CPU so a library built on another machine is never
loaded.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import platform
import subprocess

import numpy as np

from . import fem_oracle as fo  # noqa: F401  (package import)

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "cfem.c")
_lib = None

KIND = {"p1": 1, "p1k": 1, "p2": 2, "vp2": 3, "p3": 4}


def _cpu_fingerprint() -> str:
    model = platform.processor() or ""
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name") or line.startswith("flags"):
                    model += line
    except OSError:
        pass
    return hashlib.sha1(model.encode()).hexdigest()[:10]


def library_path() -> str:
    return os.path.join(_HERE, "_build", f"libcfem_{_cpu_fingerprint()}.so")


def build(force: bool = False) -> str:
    out = library_path()
    if force or not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(_SRC):
        os.makedirs(os.path.dirname(out), exist_ok=True)
        tmp = out + f".tmp{os.getpid()}"
        subprocess.check_call(["gcc", "-O3", "-march=native", "-fPIC", "-shared", "-pthread",
                               "-o", tmp, _SRC, "-lm"])
        os.replace(tmp, out)
    return out


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(build())
        vp, i64, i32, dbl = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double
        L.cfem_plan_create.restype = vp
        L.cfem_plan_create.argtypes = [i32, vp, i64, i32, i64]
        L.cfem_plan_destroy.argtypes = [vp]
        L.cfem_plan_total_cells.restype = i64
        L.cfem_plan_total_cells.argtypes = [vp]
        L.cfem_set_tables.argtypes = [vp, vp, vp]
        L.cfem_set_tables_p3.argtypes = [vp, vp]
        L.cfem_assemble_matrix.argtypes = [vp, i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, dbl, vp, i64]
        L.cfem_assemble_vector.argtypes = [vp, i32, vp, vp, vp, i32, vp, vp]
        L.cfem_apply_lifting.argtypes = [vp, i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, dbl, vp]
        L.cfem_set_bc.argtypes = [vp, vp, i64, vp, vp, dbl]
        L.cfem_matrix_bound.argtypes = [vp, i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, dbl, dbl]
        L.cfem_rhs_bound.argtypes = [vp, i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, dbl, vp, dbl, dbl]
        L.cfem_pattern_build.restype = i64
        L.cfem_pattern_build.argtypes = [vp, vp, i32, i32, i64, ctypes.POINTER(vp), ctypes.POINTER(vp)]
        L.cfem_free.argtypes = [vp]
        r2w = np.ascontiguousarray(fo.ref_grad_tensor(2, True))
        r2 = np.ascontiguousarray(fo.ref_grad_tensor(2, False))
        w2 = np.ascontiguousarray(fo.ref_basis_integrals(2))
        r3 = np.ascontiguousarray(fo.ref_grad_tensor(3, False))
        w3 = np.ascontiguousarray(fo.ref_basis_integrals(3))
        L._tables = (r2w, r2, w2, r3, w3)
        L.cfem_set_tables(r2w.ctypes.data, r2.ctypes.data, w2.ctypes.data)
        L.cfem_set_tables_p3(r3.ctypes.data, w3.ctypes.data)
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def pattern(dofs, num_blocks, bs=1, nthreads=None):
    """CSR pattern (row_ptr, col) of a cell integral on one dofmap, built by
    row-owning threads: DOLFINx's sorted unique block columns per block row,
    unrolled to scalar rows as cpp/cudolfinx/la/petsc.cpp:45-65 does (the same
    arrays as fem_oracle.sparsity)."""
    L = lib()
    d = np.ascontiguousarray(dofs, dtype=np.int32)
    nthreads = nthreads or os.cpu_count() or 1
    plan = L.cfem_plan_create(nthreads, d.ctypes.data, d.shape[0], d.shape[1], num_blocks)
    try:
        rp, cl = ctypes.c_void_p(), ctypes.c_void_p()
        nnz = L.cfem_pattern_build(plan, d.ctypes.data, d.shape[1], bs, num_blocks, ctypes.byref(rp),
                                   ctypes.byref(cl))
        if nnz < 0:
            raise ValueError("pattern has more than 2^31-1 entries")
        nrows = num_blocks * bs
        row_ptr = np.ctypeslib.as_array((ctypes.c_int32 * (nrows + 1)).from_address(rp.value)).copy()
        col = np.ctypeslib.as_array((ctypes.c_int32 * max(nnz, 1)).from_address(cl.value))[:nnz].copy()
        L.cfem_free(rp)
        L.cfem_free(cl)
    finally:
        L.cfem_plan_destroy(plan)
    return row_ptr, col


class CpuAssembler:
    """Row-owning multithreaded CPU assembly of one problem from fem_oracle.build_problem."""

    def __init__(self, P, row_ptr, col, nthreads=None):
        self.L = lib()
        self.P = P
        self.kind = KIND[P["kind"]]
        self.nthreads = nthreads or os.cpu_count() or 1
        self.coords = np.ascontiguousarray(P["coords"], dtype=np.float64)
        self.cells = np.ascontiguousarray(P["cells"], dtype=np.int32)
        self.dofs = np.ascontiguousarray(P["dofs"], dtype=np.int32)
        self.bs = P["bs"]
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        nscal = P["ndof"] * self.bs
        self.markers = np.zeros(nscal, dtype=np.uint8)
        self.markers[P["bc_dofs"]] = 1
        self.bc_dofs = np.ascontiguousarray(P["bc_dofs"], dtype=np.int32)
        kind = P["kind"]
        if kind == "vp2":
            self.c0, self.c1 = np.ascontiguousarray(P["lam"]), np.ascontiguousarray(P["mu"])
            self.f = np.ascontiguousarray(P["f"], dtype=np.float64).reshape(-1)
        else:
            self.c0 = None if P.get("k") is None else np.ascontiguousarray(P["k"], dtype=np.float64)
            self.c1 = None
            self.f = np.ascontiguousarray(P["f"], dtype=np.float64)
        self.g = np.ascontiguousarray(P["g"], dtype=np.float64)
        self.plan = self.L.cfem_plan_create(self.nthreads, self.dofs.ctypes.data, len(self.cells),
                                            self.dofs.shape[1], P["ndof"])
        self.values = np.zeros(len(self.col))
        self.b = np.zeros(nscal)

    def close(self):
        if self.plan:
            self.L.cfem_plan_destroy(self.plan)
            self.plan = None

    __del__ = close

    def assemble_matrix(self, diagonal=1.0):
        self.L.cfem_assemble_matrix(self.plan, self.kind, _p(self.coords), _p(self.cells), _p(self.dofs),
                                    self.bs, _p(self.c0), _p(self.c1), _p(self.row_ptr), _p(self.col),
                                    _p(self.markers), _p(self.values), diagonal, _p(self.bc_dofs),
                                    len(self.bc_dofs))
        return self.values

    def matrix_bound(self, rtol=fo.PARITY_RTOL, frel=fo.PARITY_FREL):
        """Per-slot parity bound of assemble_matrix (fem_oracle.matrix_bound)."""
        out = np.empty(len(self.col))
        self.L.cfem_matrix_bound(self.plan, self.kind, _p(self.coords), _p(self.cells), _p(self.dofs), self.bs,
                                 _p(self.c0), _p(self.c1), _p(self.row_ptr), _p(self.col), _p(self.markers),
                                 _p(out), rtol, frel)
        return out

    def rhs_bound(self, scale=1.0, rtol=fo.PARITY_RTOL, frel=fo.PARITY_FREL):
        """Per-entry parity bound of assemble_rhs (vector_bound + lifting_bound,
        0 on the set_bc rows)."""
        out = np.empty(len(self.b))
        self.L.cfem_rhs_bound(self.plan, self.kind, _p(self.coords), _p(self.cells), _p(self.dofs), self.bs,
                              _p(self.f), _p(self.c0), _p(self.c1), _p(self.markers), _p(self.g), None, scale,
                              _p(out), rtol, frel)
        out[self.bc_dofs] = 0.0
        return out

    def assemble_rhs(self, scale=1.0):
        self.L.cfem_assemble_vector(self.plan, self.kind, _p(self.coords), _p(self.cells), _p(self.dofs),
                                    self.bs, _p(self.f), _p(self.b))
        self.L.cfem_apply_lifting(self.plan, self.kind, _p(self.coords), _p(self.cells), _p(self.dofs),
                                  self.bs, _p(self.c0), _p(self.c1), _p(self.markers), _p(self.g), None,
                                  scale, _p(self.b))
        self.L.cfem_set_bc(_p(self.b), _p(self.bc_dofs), len(self.bc_dofs), _p(self.g), None, scale)
        return self.b
