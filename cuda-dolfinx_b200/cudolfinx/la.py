"""Device matrix/vector handles (mirror python/cudolfinx/la.py:9-75).

In the reference these wrap PETSc AIJCUSPARSE / VECCUDA objects whose device
arrays the kernels write (cpp/cudolfinx/la/CUDASeqMatrix.cpp:435-457,
CUDAVector.cpp:348-365).  Here the device arrays are torch tensors (device
memory only; torch is not on the compute path) and the CSR pattern belongs to
an engine sparsity object.  ``.mat`` / ``.vector`` hand out what a PETSc-free
consumer needs: ``mat`` is a host scipy CSR copy, ``device_csr()`` gives the
device arrays (row_ptr, col, values) for a GPU solver, and ``vector`` is the
device tensor.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib


class Sparsity:
    """Engine CSR pattern (create_cuda_matrix, cpp/cudolfinx/la/petsc.cpp:14-151)."""

    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.handle = handle
        r, c, n = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _lib.check(_lib.lib.fe_sparsity_info(handle, ctypes.byref(r), ctypes.byref(c), ctypes.byref(n)),
                   "fe_sparsity_info")
        self.num_rows, self.num_cols, self.nnz = r.value, c.value, n.value

    @classmethod
    def build(cls, ctx, dofmap0, dofmap1, on_device: bool = True):
        """CSR pattern of the cell integral (create_cuda_matrix, la/petsc.cpp:14-151);
        built on the device by default, on the host with ``on_device=False``
        (the same arrays, bit for bit)."""
        h = _lib.out_handle()
        if on_device:
            _lib.check(_lib.lib.fe_sparsity_build_device(dofmap0.handle, dofmap1.handle, ctx.stream(), h),
                       "fe_sparsity_build_device")
        else:
            _lib.check(_lib.lib.fe_sparsity_build(dofmap0.handle, dofmap1.handle, h), "fe_sparsity_build")
        return cls(ctx, h.value)

    @classmethod
    def build_block(cls, ctx, parts, num_rows: int, num_cols: int):
        """Monolithic pattern of a block form (create_cuda_matrix_block,
        cpp/cudolfinx/fem/petsc.h:39-107): ``parts`` = [(row dofmap, column
        dofmap, row offset, column offset)], one per non-empty block."""
        n = len(parts)
        rows = (ctypes.c_void_p * max(1, n))(*[p[0].handle for p in parts])
        cols = (ctypes.c_void_p * max(1, n))(*[p[1].handle for p in parts])
        roff = np.ascontiguousarray([p[2] for p in parts] or [0], dtype=np.int64)
        coff = np.ascontiguousarray([p[3] for p in parts] or [0], dtype=np.int64)
        h = _lib.out_handle()
        _lib.check(_lib.lib.fe_sparsity_build_block(ctx.handle, n, rows, cols, roff.ctypes.data, coff.ctypes.data,
                                                    int(num_rows), int(num_cols), h), "fe_sparsity_build_block")
        return cls(ctx, h.value)

    @classmethod
    def build_forms(cls, ctx, forms):
        """Pattern of a sum of bilinear forms on the same spaces: the union of
        their cell / interior-facet couplings (create_sparsity_pattern of a
        form with several integrals)."""
        hs = [h for f in forms for h in f._integral_handles()]
        n = len(hs)
        tab = (ctypes.c_void_p * n)(*hs)
        h = _lib.out_handle()
        _lib.check(_lib.lib.fe_sparsity_build_forms(n, tab, h), "fe_sparsity_build_forms")
        return cls(ctx, h.value)

    @classmethod
    def from_csr(cls, ctx, row_ptr, col, num_cols):
        rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
        cl = np.ascontiguousarray(col, dtype=np.int32)
        h = _lib.out_handle()
        _lib.check(_lib.lib.fe_sparsity_create(ctx.handle, rp.ctypes.data, cl.ctypes.data if cl.size else None,
                                               len(rp) - 1, num_cols, h), "fe_sparsity_create")
        return cls(ctx, h.value)

    def to_host(self):
        rp = np.empty(self.num_rows + 1, dtype=np.int32)
        cl = np.empty(self.nnz, dtype=np.int32)
        _lib.check(_lib.lib.fe_sparsity_copy_to_host(self.handle, rp.ctypes.data, cl.ctypes.data if self.nnz else None),
                   "fe_sparsity_copy_to_host")
        return rp, cl

    def device_arrays(self):
        """(row_ptr, col) as int32 device tensors viewing the engine's arrays."""
        rp, cl = ctypes.c_void_p(), ctypes.c_void_p()
        _lib.check(_lib.lib.fe_sparsity_device_arrays(self.handle, ctypes.byref(rp), ctypes.byref(cl)),
                   "fe_sparsity_device_arrays")
        return (_DeviceView(rp.value, self.num_rows + 1, "<i4", self).tensor(),
                _DeviceView(cl.value, self.nnz, "<i4", self).tensor())

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self.handle = None
            release = getattr(_lib, "release", None)  # None during interpreter teardown
            if release is not None:
                release("fe_sparsity_destroy", h)


class _DeviceView:
    """__cuda_array_interface__ view of engine-owned device memory."""

    def __init__(self, ptr, n, typestr, owner):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr or 0, False),
                                         "version": 3, "strides": None}
        self._owner = owner

    def tensor(self):
        return torch.as_tensor(self, device="cuda")


class CUDAVector:
    """Vector on the device."""

    def __init__(self, ctx, n: int, values: torch.Tensor | None = None):
        self._ctx = ctx
        self.size = n
        self._values = values if values is not None else torch.zeros(n, dtype=torch.float64,
                                                                      device=ctx.torch_device)
        self._read_done = None  # event of a pending copy_to_host

    def copy_to_host(self, out: torch.Tensor | None = None) -> torch.Tensor:
        """Asynchronous device -> host copy into `out` (a pinned CPU float64
        tensor of `size` values; allocated pinned when None), on the context's
        download stream once the work already queued on the current stream is
        done; it overlaps work queued afterwards.  The assembler's next writes
        into this vector wait for it; synchronise before reading `out` (e.g.
        torch.cuda.synchronize()), and order other writes to ``vector`` after
        ctx.join_transfers()."""
        if out is None:
            out = torch.empty(self.size, dtype=torch.float64, pin_memory=True)
        if 8 * self.size < (1 << 20):
            # small vectors: on the current stream (an event round trip would
            # cost more than the overlap)
            out.copy_(self._values, non_blocking=True)
            return out
        dn = self._ctx.download_stream()
        dn.wait_stream(self._ctx.torch_stream())
        with torch.cuda.stream(dn):
            out.copy_(self._values, non_blocking=True)
        self._values.record_stream(dn)
        ev = torch.cuda.Event()
        ev.record(dn)
        self._read_done = ev
        return out

    def _before_write(self):
        """Order a write on the current stream after a pending copy_to_host."""
        if self._read_done is not None:
            self._ctx.torch_stream().wait_event(self._read_done)
            self._read_done = None

    @property
    def vector(self) -> torch.Tensor:
        """The device values (stand-in for the PETSc Vec of the reference)."""
        return self._values

    @property
    def array(self) -> np.ndarray:
        return self.to_host()

    def to_host(self) -> np.ndarray:
        """Copy device values to a host array (CUDAVector::copy_vector_values_to_host)."""
        self._ctx.join_transfers()
        torch.cuda.current_stream(self._ctx.device).synchronize()
        return self._values.cpu().numpy()


class CUDAMatrix:
    """CSR matrix on the device: engine pattern + torch value array."""

    def __init__(self, ctx, sparsity: Sparsity, values: torch.Tensor | None = None):
        self._ctx = ctx
        self.sparsity = sparsity
        self._values = values if values is not None else torch.zeros(sparsity.nnz, dtype=torch.float64,
                                                                     device=ctx.torch_device)

    @property
    def values(self) -> torch.Tensor:
        return self._values

    def assemble(self):
        """Finalise: wait for the assembly and surface device error words
        (the reference calls MatAssemblyBegin/End here, wrappers/fem.cpp:176-181)."""
        self._ctx.synchronize()

    def device_csr(self):
        rp, cl = self.sparsity.device_arrays()
        return rp, cl, self._values

    @property
    def mat(self):
        """Host scipy.sparse CSR copy (PETSc-free stand-in for the reference's petsc4py Mat)."""
        import scipy.sparse as sp
        self.assemble()
        rp, cl = self.sparsity.to_host()
        return sp.csr_matrix((self._values.cpu().numpy(), cl, rp),
                             shape=(self.sparsity.num_rows, self.sparsity.num_cols))
