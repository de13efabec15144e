"""CUDAForm and ``form()`` (mirrors python/cudolfinx/form.py:26-105, 227-262).

The reference compiles a UFL form with FFCx, scrapes the generated
tabulate_tensor C bodies and NVRTC-compiles them into its kernel templates.
Here a ``FormSpec`` (cudolfinx.fem) selects one of the engine's built-in
element kernels, compiled ahead of time for sm_100a.  As in the reference the
device mesh is created once per mesh (``_create_mesh_on_device`` is cached,
form.py:252-262) and dofmaps once per function space.
"""
from __future__ import annotations

import ctypes
import typing

import numpy as np

from . import _lib
from .context import get_cuda_context
from .fem import FormSpec, Function, FunctionSpace

DEFAULT_CUDA_JIT_ARGS = {"max_threads_per_block": 1024, "min_blocks_per_multiprocessor": 1}

_mesh_cache: dict[int, "DeviceMesh"] = {}
_dofmap_cache: dict[int, "DeviceDofMap"] = {}


class DeviceMesh:
    def __init__(self, ctx, mesh):
        self.ctx = ctx
        self.mesh = mesh
        h = _lib.out_handle()
        x, c = mesh.geometry_x, mesh.cells
        _lib.check(_lib.lib.fe_mesh_create(ctx.handle, x.ctypes.data, len(x), c.ctypes.data, len(c), 4, h),
                   "fe_mesh_create")
        self.handle = h.value

    def __del__(self):
        if getattr(self, "handle", None):
            _lib.lib.fe_mesh_destroy(self.handle)
            self.handle = None


class DeviceDofMap:
    def __init__(self, ctx, V: FunctionSpace):
        self.ctx = ctx
        self.V = V
        h = _lib.out_handle()
        d = np.ascontiguousarray(V.dofs, dtype=np.int32)
        _lib.check(_lib.lib.fe_dofmap_create(ctx.handle, d.ctypes.data, d.shape[0], d.shape[1], V.bs,
                                             V.num_nodes, h), "fe_dofmap_create")
        self.handle = h.value

    def __del__(self):
        if getattr(self, "handle", None):
            _lib.lib.fe_dofmap_destroy(self.handle)
            self.handle = None


def _create_mesh_on_device(ctx, mesh) -> DeviceMesh:
    m = _mesh_cache.get(id(mesh))
    if m is None or m.mesh is not mesh:
        m = DeviceMesh(ctx, mesh)
        _mesh_cache[id(mesh)] = m
    return m


def release_device_caches(mesh=None):
    """Drop cached device meshes and dofmaps: all of them, or those of `mesh`.
    Objects still referenced by live forms stay alive through those forms."""
    for k, m in list(_mesh_cache.items()):
        if mesh is None or m.mesh is mesh:
            _mesh_cache.pop(k, None)
    for k, d in list(_dofmap_cache.items()):
        if mesh is None or d.V.mesh is mesh:
            _dofmap_cache.pop(k, None)


def device_dofmap(ctx, V: FunctionSpace) -> DeviceDofMap:
    d = _dofmap_cache.get(id(V))
    if d is None or d.V is not V:
        d = DeviceDofMap(ctx, V)
        _dofmap_cache[id(V)] = d
    return d


class CUDAForm:
    """CUDA wrapper of a built-in form (the reference wraps a dolfinx.fem.Form)."""

    def __init__(self, form: FormSpec, jit_args: typing.Optional[dict] = None):
        if not isinstance(form, FormSpec):
            raise TypeError(f"Expected a cudolfinx.fem.FormSpec, got '{type(form)}'")
        self._ctx = get_cuda_context()
        self._spec = form
        self._cuda_mesh = _create_mesh_on_device(self._ctx, form.mesh)
        self._dofmaps = [device_dofmap(self._ctx, V) for V in form.function_spaces]
        self._jit_args = dict(DEFAULT_CUDA_JIT_ARGS, **(jit_args or {}))
        h = _lib.out_handle()
        trial = self._dofmaps[1].handle if form.rank == 2 else None
        test = self._dofmaps[0].handle if form.rank >= 1 else None
        _lib.check(_lib.lib.fe_form_create(self._ctx.handle, _lib.FORM[form.kind], self._cuda_mesh.handle,
                                           test, trial, h), "fe_form_create")
        self._handle = h.value
        if form.facets is not None:
            fc = np.ascontiguousarray(form.facets, dtype=np.int32)
            self._facets = fc
            _lib.check(_lib.lib.fe_form_set_facets(self._handle, fc.ctypes.data, len(fc)), "fe_form_set_facets")
        if form.precision == "fp32":
            _lib.check(_lib.lib.fe_form_set_precision(self._handle, _lib.PREC_FP32), "fe_form_set_precision")
        self._bound_sparsity = None
        self._coef_refs: list = [None] * len(form.coefficients)
        self._aux_dofmaps: dict = {}
        self.to_device()

    # -- coefficients -------------------------------------------------------
    def _set_coefficient(self, i: int, c):
        ctx = self._ctx
        ncomp = 3 if self._spec.kind in ("VP2_LOAD", "VP2_FACET_LOAD") else 1
        C = self._spec.mesh.num_cells
        if isinstance(c, Function):
            V = c.function_space
            vals = np.ascontiguousarray(c.x.array, dtype=np.float64)
            if V.family == "DG":
                kind, cmap = _lib.COEFF_DG0, None
            elif V.degree == 1 and V.bs == 1:
                kind, cmap = _lib.COEFF_P1, device_dofmap(ctx, V)
                self._aux_dofmaps[i] = cmap
            elif V.degree == 2 and V.bs == 1 and self._spec.kind == "P2_ENERGY":
                kind, cmap = _lib.COEFF_P2, device_dofmap(ctx, V)
                self._aux_dofmaps[i] = cmap
            else:
                raise ValueError("coefficients must be constants, DG0 or scalar P1 Functions")
            self._coef_refs[i] = vals
            _lib.check(_lib.lib.fe_form_set_coefficient(self._handle, i, kind, cmap.handle if cmap else None,
                                                        vals.ctypes.data, len(vals), 0, ctx.stream()),
                       "fe_form_set_coefficient")
            return
        if hasattr(c, "data_ptr"):  # device tensor: DG0 values read in place
            if c.numel() != C * ncomp:
                raise ValueError("device coefficient arrays must hold one value per cell (DG0)")
            self._coef_refs[i] = c
            _lib.check(_lib.lib.fe_form_set_coefficient(self._handle, i, _lib.COEFF_DG0, None, c.data_ptr(),
                                                        c.numel(), 1, ctx.stream()), "fe_form_set_coefficient")
            return
        arr = np.atleast_1d(np.asarray(c, dtype=np.float64)).ravel()
        if arr.size == ncomp:
            kind = _lib.COEFF_CONSTANT
        elif arr.size == C * ncomp:
            kind = _lib.COEFF_DG0
        else:
            raise ValueError(f"coefficient of size {arr.size}: expected {ncomp} (constant) or "
                             f"{C * ncomp} (DG0) values")
        arr = np.ascontiguousarray(arr)
        self._coef_refs[i] = arr
        _lib.check(_lib.lib.fe_form_set_coefficient(self._handle, i, kind, None, arr.ctypes.data, arr.size, 0,
                                                    ctx.stream()), "fe_form_set_coefficient")

    def to_device(self, coefficients: typing.Optional[list] = None):
        """Copy host-side coefficient values to the device (CUDAForm.h:195-199).
        With ``coefficients`` given, only those Functions are re-uploaded."""
        for i, c in enumerate(self._spec.coefficients):
            if coefficients is None or any(c is q for q in coefficients):
                self._set_coefficient(i, c)

    # -- pattern binding ----------------------------------------------------
    def _bind(self, sparsity):
        if self._bound_sparsity is not sparsity:
            _lib.check(_lib.lib.fe_form_bind_sparsity(self._handle, sparsity.handle, self._ctx.stream()),
                       "fe_form_bind_sparsity")
            self._bound_sparsity = sparsity

    # -- properties mirroring the reference --------------------------------
    @property
    def cuda_form(self):
        return self._handle

    @property
    def cuda_mesh(self):
        return self._cuda_mesh

    @property
    def dolfinx_form(self) -> FormSpec:
        return self._spec

    @property
    def function_spaces(self):
        return self._spec.function_spaces

    @property
    def rank(self) -> int:
        return self._spec.rank

    def __del__(self):
        if getattr(self, "_handle", None):
            _lib.lib.fe_form_destroy(self._handle)
            self._handle = None


def form(form: typing.Union[FormSpec, typing.Iterable[FormSpec]], restriction=None,
         cuda_jit_args: typing.Optional[dict] = None, **kwargs):
    """Create a CUDAForm (or a list of them) from built-in form specs
    (mirrors cudolfinx.form, python/cudolfinx/form.py:227-249).  Block forms
    and restrictions are not part of this engine."""
    if restriction is not None:
        raise NotImplementedError("restricted/block forms are outside this engine")
    if isinstance(form, FormSpec):
        return CUDAForm(form, cuda_jit_args)
    return [CUDAForm(f, cuda_jit_args) for f in form]
