"""CUDAAssembler (mirrors python/cudolfinx/assemble.py:40-380).

Same method names, arguments and semantics as the reference for the
single-form path: ``assemble_matrix`` zeroes (zero=True), assembles with BC
rows/columns skipped and sets ``diagonal`` on owned BC rows;
``assemble_vector``; ``apply_lifting`` (b -= scale A (g - x0)); ``set_bc``
(b[bc] = scale (g - x0)).  Differences: work is asynchronous on torch's
current stream (the reference synchronises after every kernel);
``diagonal`` is honoured (the reference's binding always uses 1.0,
wrappers/fem.cpp:274); ``scale`` stays double (the reference's binding
takes a C float, wrappers/fem.cpp:335, 361).  Block forms (``cudolfinx.form``
of a list / list of lists, optionally restricted) assemble into one monolithic
matrix / vector with ``assemble_matrix_block`` / ``assemble_vector_block``
(assemble.py:112-202).  ``assemble_scalar`` returns the functional's value with
a fixed-order reduction.  Additions: ``deterministic=True`` selects a
bitwise-reproducible matrix variant, ``assemble_matrix_batch`` assembles many
coefficient instances at once, and ``solve`` runs the on-device Jacobi-PCG.
"""
from __future__ import annotations

import typing

import numpy as np
import torch

from . import _lib
from .bcs import CUDADirichletBC
from .context import get_cuda_context
from .fem import DirichletBC, FunctionSpace
from .form import BlockCUDAForm, CUDAForm
from .la import CUDAMatrix, CUDAVector, Sparsity

_sparsity_cache: dict = {}


def release_sparsity_cache(mesh=None):
    """Drop cached CSR patterns: all, or those built on `mesh`."""
    for k, e in list(_sparsity_cache.items()):
        if mesh is None or e[0].V.mesh is mesh:
            _sparsity_cache.pop(k, None)


class CUDAAssembler:
    """Class for assembly on the GPU."""

    def __init__(self):
        self._ctx = get_cuda_context()

    # -- creation ------------------------------------------------------------
    def create_matrix(self, a) -> CUDAMatrix:
        """Device CSR matrix for a bilinear form (create_cuda_matrix,
        assemble.py:228-234).  ``a`` may also be a list of bilinear forms on
        the same spaces whose sum is to be assembled into one matrix (the
        integrals of one DOLFINx form, e.g. a DG cell term and its
        interior-facet jump term): the pattern is the union of their
        couplings and every form is bound to it."""
        if isinstance(a, (list, tuple)):
            forms = list(a)
            if not forms or not all(isinstance(f, CUDAForm) and f.rank == 2 for f in forms):
                raise TypeError("Expected a list of bilinear CUDAForms")
            sp = Sparsity.build_forms(self._ctx, forms)
            mat = CUDAMatrix(self._ctx, sp)
            for f in forms:
                f._bind(sp)
            return mat
        if not isinstance(a, CUDAForm):
            raise TypeError(f"Expected CUDAForm, got type '{type(a)}'.")
        if a.rank != 2:
            raise ValueError("create_matrix needs a bilinear form")
        if a._needs_union_pattern():
            # interior-facet couplings join the two cells of every facet
            sp = Sparsity.build_forms(self._ctx, [a])
            mat = CUDAMatrix(self._ctx, sp)
            a._bind(sp)
            return mat
        if a.restriction(0) is not None or a.restriction(1) is not None:
            # a restricted form is a one-block system
            sp = Sparsity.build_block(self._ctx, [(a._dofmaps[0], a._dofmaps[1], 0, 0)], a.space_size(0),
                                      a.space_size(1))
            mat = CUDAMatrix(self._ctx, sp)
            a._bind_block(sp, 0, 0)
            return mat
        key = (id(a._dofmaps[0]), id(a._dofmaps[1]))
        entry = _sparsity_cache.get(key)
        if entry is None or entry[0] is not a._dofmaps[0] or entry[1] is not a._dofmaps[1]:
            sp = Sparsity.build(self._ctx, a._dofmaps[0], a._dofmaps[1])
            entry = (a._dofmaps[0], a._dofmaps[1], sp)
            _sparsity_cache[key] = entry
        mat = CUDAMatrix(self._ctx, entry[2])
        a._bind(mat.sparsity)
        return mat

    def create_vector(self, b: CUDAForm) -> CUDAVector:
        if not isinstance(b, CUDAForm):
            raise TypeError(f"Expected CUDAForm, got type '{type(b)}'.")
        return CUDAVector(self._ctx, b.space_size(0))

    def create_matrix_block(self, a: BlockCUDAForm) -> CUDAMatrix:
        """Monolithic matrix of a block form (create_matrix_block,
        assemble.py:236-243 -> cpp/cudolfinx/fem/petsc.h:39-107); every block
        form is bound to it at its offsets."""
        if not isinstance(a, BlockCUDAForm):
            raise TypeError(f"Expected BlockCUDAForm, got type '{type(a)}'")
        parts = [(f._dofmaps[0], f._dofmaps[1], a.row_offsets[i], a.col_offsets[j])
                 for i, row in enumerate(a.forms) for j, f in enumerate(row) if f is not None]
        sp = Sparsity.build_block(self._ctx, parts, a.row_offsets[-1], a.col_offsets[-1])
        mat = CUDAMatrix(self._ctx, sp)
        self._bind_blocks(a, mat)
        return mat

    def _bind_blocks(self, a: BlockCUDAForm, mat: CUDAMatrix):
        for i, row in enumerate(a.forms):
            for j, f in enumerate(row):
                if f is not None:
                    f._bind_block(mat.sparsity, a.row_offsets[i], a.col_offsets[j])

    def create_vector_block(self, b: BlockCUDAForm) -> CUDAVector:
        """Monolithic vector of a block linear form (assemble.py:255-262)."""
        if not isinstance(b, BlockCUDAForm):
            raise TypeError(f"Expected BlockCUDAForm, got type '{type(b)}')")
        return CUDAVector(self._ctx, b.local_size)

    def pack_bcs(self, bcs: list[DirichletBC]) -> CUDADirichletBC:
        return CUDADirichletBC(self._ctx, bcs)

    def pack_coefficients(self, a: CUDAForm, coefficients: typing.Optional[list] = None):
        """Kept for API parity (assemble.py:274-285).  The element kernels
        gather coefficient values from their device arrays directly, so there
        is no packed copy to refresh; host changes reach the device through
        ``CUDAForm.to_device``, which assemble_matrix / assemble_vector call."""
        if not isinstance(a, CUDAForm):
            raise TypeError(f"Expected CUDAForm, got type '{type(a)}'.")

    def _bc_collection(self, bcs) -> CUDADirichletBC:
        if isinstance(bcs, CUDADirichletBC):
            return bcs
        if isinstance(bcs, (list, tuple)):
            return self.pack_bcs(list(bcs))
        raise TypeError(f"Expected either a list of DirichletBC's or a CUDADirichletBC, got '{type(bcs)}'")

    # -- assembly ------------------------------------------------------------
    def assemble_matrix(self, a: CUDAForm, mat: typing.Optional[CUDAMatrix] = None, bcs=(), diagonal: float = 1.0,
                        constants=None, coeffs=None, zero: bool = True, deterministic: bool = False,
                        variant: str = "auto") -> CUDAMatrix:
        """Assemble a bilinear form into a device CSR matrix (not finalised).

        ``variant``: "auto" (block variant for P1 on meshes of >= 2^20 cells,
        coalesced scatter for P2 stiffness, vector-P2 elasticity and FP64 P3
        stiffness, atomic scatter otherwise),
        "deterministic" (bitwise reproducible: ordered tile gather for P1/P2,
        sorted-slot otherwise), "atomic" (FP64-atomic scatter, one thread's
        reductions per cell), "coalesced" (P2, vector P2, FP64 P3: a warp's
        reductions issued row by row, consecutive lanes on consecutive columns),
        "grouped" (P2: one reduction per distinct
        slot of 48-cell groups), "sorted-slot" (global sorted-slot
        reduction), "block" (Morton cell blocks combined in shared memory,
        P1/P2), "tile" (owner-computes row tiles, P1/P2), "row-gather" (P1),
        "atomic-full" (atomic scatter into both triangles, the reference's
        scheme).
        ``deterministic=True`` is the same as variant="deterministic"."""
        if variant not in _lib.VARIANT_FLAGS:
            raise ValueError(f"unknown variant {variant!r}; expected one of {sorted(_lib.VARIANT_FLAGS)}")
        if not isinstance(a, CUDAForm):
            raise TypeError(f"Expected CUDAForm, got '{type(a)}'")
        if mat is None:
            mat = self.create_matrix(a)
        else:
            a._bind(mat.sparsity)
        col = self._bc_collection(bcs)
        bc0 = col._get_cpp_bcs(a.function_spaces[0], a.restriction(0))
        bc1 = col._get_cpp_bcs(a.function_spaces[1], a.restriction(1))
        # as the reference (assemble.py:100-103): always copy host coefficients to the device
        a.to_device()
        self.pack_coefficients(a, coeffs)
        flags = (_lib.ASM_DETERMINISTIC if deterministic else 0) | _lib.VARIANT_FLAGS[variant]
        # a form with several integrals: the first zeroes, the others add
        for q, h in enumerate(a._integral_handles()):
            _lib.check(_lib.lib.fe_assemble_matrix(h, mat.values.data_ptr(), bc0.handle if bc0 else None,
                                                   bc1.handle if bc1 else None, float(diagonal),
                                                   flags | (_lib.ASM_ZERO if (zero and q == 0) else 0),
                                                   self._ctx.stream()), "fe_assemble_matrix")
        a._mark_used()
        mat._bcs = col  # keep device BC data alive while the work is queued
        return mat

    def assemble_matrix_batch(self, a: CUDAForm, coefficients, mats: typing.Optional[list] = None, bcs=(),
                              diagonal: float = 1.0, zero: bool = True) -> list:
        """Assemble many instances of a P1/P2 stiffness form that differ only
        in a DG0 coefficient, in one batched launch (no counterpart in the
        reference, which assembles one form per call).

        ``coefficients``: a sequence of device float64 tensors of length
        num_cells, or one (instances, num_cells) tensor.  ``mats``: CUDAMatrix
        objects sharing the form's pattern (created when None).  Element
        tensors are FP32 and slot sums FP64 in a fixed order, so results are
        bitwise reproducible; BC semantics match ``assemble_matrix``."""
        if not isinstance(a, CUDAForm):
            raise TypeError(f"Expected CUDAForm, got '{type(a)}'")
        if isinstance(coefficients, torch.Tensor) and coefficients.dim() == 2:
            coefficients = list(coefficients.unbind(0))
        coefficients = list(coefficients)
        if not coefficients and not mats:
            return []
        ncells = a._spec.mesh.num_cells
        for k in coefficients:
            if not (isinstance(k, torch.Tensor) and k.is_cuda and k.dtype == torch.float64 and k.is_contiguous()
                    and k.numel() == ncells):
                raise ValueError("each coefficient must be a contiguous float64 device tensor of num_cells values")
        if mats is None:
            first = self.create_matrix(a)
            mats = [first] + [CUDAMatrix(self._ctx, first.sparsity) for _ in coefficients[1:]]
        elif len(mats) != len(coefficients):
            raise ValueError("need one matrix per coefficient instance")
        if mats:
            a._bind(mats[0].sparsity)
            for m in mats[1:]:
                if m.sparsity is not mats[0].sparsity:
                    raise ValueError("all matrices of a batch must share one sparsity pattern")
        col = self._bc_collection(bcs)
        bc0 = col._get_cpp_bcs(a.function_spaces[0])
        bc1 = col._get_cpp_bcs(a.function_spaces[1])
        a.to_device()
        import ctypes
        n = len(coefficients)
        ktab = (ctypes.c_void_p * max(1, n))(*[k.data_ptr() for k in coefficients])
        vtab = (ctypes.c_void_p * max(1, n))(*[m.values.data_ptr() for m in mats])
        _lib.check(_lib.lib.fe_assemble_matrix_batch(a.cuda_form, n, ktab, vtab, bc0.handle if bc0 else None,
                                                     bc1.handle if bc1 else None, float(diagonal),
                                                     _lib.ASM_ZERO if zero else 0, self._ctx.stream()),
                   "fe_assemble_matrix_batch")
        for m in mats:
            m._bcs = col
        return mats

    def assemble_matrix_block(self, a: BlockCUDAForm, mat: typing.Optional[CUDAMatrix] = None, bcs=None,
                              coeffs=None, constants=None, zero: bool = True, diagonal: float = 1.0) -> CUDAMatrix:
        """Assemble a block form into one monolithic matrix (assemble.py:112-134):
        zero it once, then add every block at its offsets.  ``bcs``: a list of
        lists (the BCs of block (i, j), as the reference takes them), or one flat
        list of DirichletBCs (or a CUDADirichletBC) applied to every block by
        function space (rows on the block's test space, columns on its trial
        space); owned BC rows get ``diagonal`` on the monolithic diagonal."""
        if not isinstance(a, BlockCUDAForm):
            raise TypeError(f"Expected BlockCUDAForm, got '{type(a)}'")
        if mat is None:
            mat = self.create_matrix_block(a)
        else:
            self._bind_blocks(a, mat)
        if zero:
            _lib.check(_lib.lib.fe_zero_entries(mat.values.data_ptr(), mat.sparsity.nnz, self._ctx.stream()),
                       "fe_zero_entries")
        nested = isinstance(bcs, (list, tuple)) and len(bcs) > 0 and isinstance(bcs[0], (list, tuple))
        flat = None if (bcs is None or nested) else self._bc_collection(bcs)
        for i, row in enumerate(a.forms):
            for j, f in enumerate(row):
                if f is None:
                    continue
                _bcs = (bcs[i][j] if nested else flat) if bcs is not None else []
                _coeffs = coeffs[i][j] if coeffs is not None else None
                self.assemble_matrix(f, mat, bcs=_bcs, coeffs=_coeffs, zero=False, diagonal=diagonal,
                                     variant="atomic")
        return mat

    def assemble_vector_block(self, b: BlockCUDAForm, vec: typing.Optional[CUDAVector] = None, constants=None,
                              coeffs=None, zero: bool = True) -> CUDAVector:
        """Assemble a block linear form into one vector, block i at offsets[i]
        (assemble.py:168-202)."""
        if not isinstance(b, BlockCUDAForm):
            raise TypeError(f"Expected BlockCUDAForm, got '{type(b)}'")
        if vec is None:
            vec = self.create_vector_block(b)
        n = len(b.forms)
        _coeffs = [None] * n if coeffs is None else coeffs
        if len(_coeffs) != n:
            raise ValueError(f"Expected coeffs to be None or a list of length: '{n}', got '{len(_coeffs)}' instead!")
        vec._before_write()
        if zero:
            vec.vector.zero_()
        base = vec.vector.data_ptr()
        for f, off, c in zip(b.forms, b.offsets, _coeffs):
            f.to_device()
            self.pack_coefficients(f, c)
            for h in f._integral_handles():
                _lib.check(_lib.lib.fe_assemble_vector(h, base + 8 * off, 0, self._ctx.stream()),
                           "fe_assemble_vector")
            f._mark_used()
        return vec

    def assemble_scalar(self, b: CUDAForm, constants=None, coeffs=None) -> float:
        """Value of a functional (assemble.py:204-226); the reduction runs in a
        fixed order, so the value is reproducible bit for bit."""
        if not isinstance(b, CUDAForm):
            raise TypeError(f"Expected CUDAForm, got '{type(b)}'")
        if b.rank != 0:
            raise ValueError("assemble_scalar needs a functional")
        import ctypes
        b.to_device()  # assemble.py:220-222
        self.pack_coefficients(b, coeffs)
        total = 0.0
        for h in b._integral_handles():
            out = ctypes.c_double(0.0)
            _lib.check(_lib.lib.fe_assemble_scalar(h, ctypes.byref(out), self._ctx.stream()), "fe_assemble_scalar")
            total += out.value
        b._mark_used()
        return total

    def assemble_vector(self, b: CUDAForm, vec: typing.Optional[CUDAVector] = None, constants=None, coeffs=None,
                        zero: bool = True) -> CUDAVector:
        """Assemble a linear form into a device vector."""
        if not isinstance(b, CUDAForm):
            raise TypeError(f"Expected CUDAForm, got '{type(b)}'")
        if vec is None:
            vec = self.create_vector(b)
        b.to_device()  # assemble.py:156-158
        self.pack_coefficients(b, coeffs)
        vec._before_write()
        if b.part == "diagonal":
            _lib.check(_lib.lib.fe_assemble_diagonal(b._handle, vec.vector.data_ptr(), _lib.ASM_ZERO if zero else 0,
                                                     self._ctx.stream()), "fe_assemble_diagonal")
        else:
            for q, h in enumerate(b._integral_handles()):
                _lib.check(_lib.lib.fe_assemble_vector(h, vec.vector.data_ptr(),
                                                       _lib.ASM_ZERO if (zero and q == 0) else 0,
                                                       self._ctx.stream()), "fe_assemble_vector")
        b._mark_used()
        return vec

    def apply_lifting(self, b: CUDAVector, a: list[CUDAForm], bcs: list, x0: typing.Optional[list] = None,
                      scale: float = 1.0, coeffs: typing.Optional[list] = None):
        """b -= scale * A_i (g_i - x0_i) over the BC columns of each form."""
        if len(a) != len(bcs):
            raise ValueError("Lengths of forms and bcs must match!")
        if x0 is not None and len(x0) != len(a):
            raise ValueError("Lengths of forms and x0 must match!")
        if coeffs is None:
            coeffs = [None] * len(a)
        elif not len(coeffs):
            coeffs = [[] for _ in a]
        import ctypes
        keep, hf, hb, hx = [], [], [], []
        for i, (f, bc, c) in enumerate(zip(a, bcs, coeffs)):
            self.pack_coefficients(f, c)
            col = self._bc_collection(bc)
            keep.append(col)
            d = col._get_cpp_bcs(f.function_spaces[1], f.restriction(1))
            for h in f._integral_handles():  # every integral of the form lifts
                hf.append(h)
                hb.append(d.handle if d else None)
                hx.append(x0[i].vector.data_ptr() if (x0 is not None and x0[i] is not None) else None)
        n = len(hf)
        forms = (ctypes.c_void_p * max(1, n))(*hf)
        hbcs = (ctypes.c_void_p * max(1, n))(*hb)
        hx0 = (ctypes.c_void_p * max(1, n))(*hx)
        b._before_write()
        _lib.check(_lib.lib.fe_apply_lifting(b.vector.data_ptr(), n, forms, hbcs, hx0 if x0 is not None else None,
                                             float(scale), self._ctx.stream()), "fe_apply_lifting")
        for f in a:
            f._mark_used()
        b._keep = keep

    def assemble_rhs(self, L: CUDAForm, a: CUDAForm, bcs, vec: typing.Optional[CUDAVector] = None,
                     x0: typing.Optional[CUDAVector] = None, scale: float = 1.0, zero: bool = True) -> CUDAVector:
        """The right-hand side of A x = b in one call: ``assemble_vector(L)``,
        ``apply_lifting(b, [a], [bcs], [x0], scale)`` and ``set_bc(b, bcs, V,
        x0, scale)`` with V the trial space of `a`.  One kernel for the
        built-in cell forms on one space (fe_assemble_rhs), the three calls
        otherwise; the result is the same."""
        if not isinstance(L, CUDAForm) or not isinstance(a, CUDAForm):
            raise TypeError("Expected CUDAForm arguments")
        hl, ha = L._integral_handles(), a._integral_handles()
        if len(hl) != 1 or len(ha) != 1 or L.part == "diagonal":
            vec = self.assemble_vector(L, vec, zero=zero)
            self.apply_lifting(vec, [a], [bcs], None if x0 is None else [x0], scale)
            self.set_bc(vec, bcs, a.function_spaces[1], x0, scale, restriction=a.restriction(1))
            return vec
        if vec is None:
            vec = self.create_vector(L)
        L.to_device()
        a.to_device()
        self.pack_coefficients(L, None)
        self.pack_coefficients(a, None)
        col = self._bc_collection(bcs)
        d = col._get_cpp_bcs(a.function_spaces[1], a.restriction(1))
        vec._before_write()
        _lib.check(_lib.lib.fe_assemble_rhs(hl[0], ha[0], d.handle if d else None, vec.vector.data_ptr(),
                                            x0.vector.data_ptr() if x0 is not None else None, float(scale),
                                            _lib.ASM_ZERO if zero else 0, self._ctx.stream()), "fe_assemble_rhs")
        L._mark_used()
        a._mark_used()
        vec._keep_bc = col
        return vec

    def set_bc(self, b: CUDAVector, bcs, V: FunctionSpace, x0: typing.Optional[CUDAVector] = None,
               scale: float = 1.0, restriction: typing.Optional[np.ndarray] = None):
        """b[bc dofs] = scale * (g - x0) on the BCs of V (in the numbering of
        `restriction`, the kept dofs of V, when b lives on a restricted space)."""
        col = self._bc_collection(bcs)
        d = col._get_cpp_bcs(V, restriction)
        if d is None:
            return
        b._before_write()
        _lib.check(_lib.lib.fe_set_bc(b.vector.data_ptr(), b.size, d.handle,
                                      x0.vector.data_ptr() if x0 is not None else None, float(scale),
                                      self._ctx.stream()), "fe_set_bc")
        b._keep_bc = col

    # -- solve ---------------------------------------------------------------
    def solve(self, A: CUDAMatrix, b: CUDAVector, x: typing.Optional[CUDAVector] = None, rtol: float = 1e-8,
              max_iter: int = 20000, raise_on_failure: bool = True, precision: str = "fp64", block_size: int = 1,
              inner_rtol: float = 1e-4):
        """Jacobi-preconditioned CG on the device; returns (x, iterations,
        relative residual).  ``precision="mixed"``: inner iterations on an FP32
        copy of the values (``block_size=3``: in a 3x3 block-column layout, for
        vector-valued spaces), refined in FP64 to ``rtol``; iterations counts
        the inner ones."""
        import ctypes
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if x is None:
            x = CUDAVector(self._ctx, b.size)
        x._before_write()
        it, res = ctypes.c_int(0), ctypes.c_double(0.0)
        if precision == "mixed":
            ref = ctypes.c_int(0)
            st = _lib.lib.fe_pcg_solve_mixed(A.sparsity.handle, A.values.data_ptr(), b.vector.data_ptr(),
                                             x.vector.data_ptr(), float(rtol), float(inner_rtol), int(max_iter),
                                             int(block_size), ctypes.byref(it), ctypes.byref(ref), ctypes.byref(res),
                                             self._ctx.stream())
            what = "fe_pcg_solve_mixed"
        else:
            st = _lib.lib.fe_pcg_solve(A.sparsity.handle, A.values.data_ptr(), b.vector.data_ptr(),
                                       x.vector.data_ptr(), float(rtol), int(max_iter), ctypes.byref(it),
                                       ctypes.byref(res), self._ctx.stream())
            what = "fe_pcg_solve"
        if st == _lib.FE_ERR_NOT_CONVERGED and not raise_on_failure:
            return x, it.value, res.value
        _lib.check(st, what)
        return x, it.value, res.value
