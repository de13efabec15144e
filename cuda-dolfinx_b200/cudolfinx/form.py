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
import torch

from . import _lib
from .context import get_cuda_context
from .fem import FFCxForm, FormSpec, Function, FunctionSpace

DEFAULT_CUDA_JIT_ARGS = {"max_threads_per_block": 1024, "min_blocks_per_multiprocessor": 1}
# transfers of at least this size run on the context's side streams (below it
# on the current stream: for a few hundred kB the extra event round trip costs
# more than the overlap gains)
OVERLAP_MIN_BYTES = 1 << 20
# device copies per uploaded coefficient: an upload fills the copy whose last
# tracked readers are the oldest, so re-uploading a coefficient (every
# assembly call uploads its host values, as the reference does) waits for
# kernels of the calls before the last two, not for the one still running
COEF_RING = 3

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
        h = getattr(self, "handle", None)
        if h:
            self.handle = None
            release = getattr(_lib, "release", None)  # None during interpreter teardown
            if release is not None:
                release("fe_mesh_destroy", h)


class DeviceDofMap:
    """Device dofmap of V; with ``restriction`` (sorted block dofs of V that
    are kept) the cell dofs are renumbered to positions in the restriction and
    dofs outside it become -1 (CUDADofMap::update with a restriction map,
    cpp/cudolfinx/fem/CUDADofMap.cpp:199-236)."""

    def __init__(self, ctx, V: FunctionSpace, restriction: typing.Optional[np.ndarray] = None):
        self.ctx = ctx
        self.V = V
        self.restriction = None if restriction is None else np.ascontiguousarray(restriction, dtype=np.int32)
        h = _lib.out_handle()
        if self.restriction is None:
            d = np.ascontiguousarray(V.dofs, dtype=np.int32)
            self.num_blocks = V.num_nodes
            _lib.check(_lib.lib.fe_dofmap_create(ctx.handle, d.ctypes.data, d.shape[0], d.shape[1], V.bs,
                                                 V.num_nodes, h), "fe_dofmap_create")
        else:
            r = self.restriction
            if r.size and (r.min() < 0 or r.max() >= V.num_nodes or np.any(np.diff(r) <= 0)):
                raise ValueError("a restriction is a sorted list of distinct dofs of the space")
            remap = np.full(V.num_nodes, -1, dtype=np.int32)
            remap[r] = np.arange(len(r), dtype=np.int32)
            d = np.ascontiguousarray(remap[V.dofs])
            self.num_blocks = len(r)
            _lib.check(_lib.lib.fe_dofmap_create_restricted(ctx.handle, d.ctypes.data, d.shape[0], d.shape[1],
                                                            V.bs, len(r), h), "fe_dofmap_create_restricted")
        self.handle = h.value

    @property
    def size(self) -> int:
        """Scalar dofs of the (restricted) space."""
        return self.num_blocks * self.V.bs

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self.handle = None
            release = getattr(_lib, "release", None)  # None during interpreter teardown
            if release is not None:
                release("fe_dofmap_destroy", h)


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

    def __init__(self, form: FormSpec, jit_args: typing.Optional[dict] = None, part: typing.Optional[str] = None):
        if not isinstance(form, FormSpec):
            raise TypeError(f"Expected a cudolfinx.fem.FormSpec, got '{type(form)}'")
        if part not in (None, "full", "diagonal"):
            raise ValueError(f"unknown form part '{part}' (expected 'full' or 'diagonal')")
        if part == "diagonal" and (form.rank != 2 or form.facets is not None
                                   or form.function_spaces[0] is not form.function_spaces[1]):
            raise ValueError("the diagonal part is offered for cell bilinear forms on one space")
        self._ctx = get_cuda_context()
        self._spec = form
        # "diagonal": the form is the matrix diagonal as a linear form on the
        # test space (FFCx's "part" option, as passed by the reference through
        # form_compiler_options)
        self._part = "diagonal" if part == "diagonal" else "full"
        self._cuda_mesh = _create_mesh_on_device(self._ctx, form.mesh)
        self._dofmaps = [device_dofmap(self._ctx, V) for V in form.function_spaces]
        self._jit_args = dict(DEFAULT_CUDA_JIT_ARGS, **(jit_args or {}))
        self._handle = None
        self._create_handle()

    def _create_handle(self):
        """(Re)create the engine form on the current dofmaps."""
        form = self._spec
        if self._handle:
            _lib.lib.fe_form_destroy(self._handle)
            self._handle = None
        h = _lib.out_handle()
        trial = self._dofmaps[1].handle if form.rank == 2 else None
        test = self._dofmaps[0].handle if form.rank >= 1 else None
        _lib.check(_lib.lib.fe_form_create(self._ctx.handle, _lib.FORM[form.kind], self._cuda_mesh.handle,
                                           test, trial, h), "fe_form_create")
        self._handle = h.value
        if form.facets is not None:
            fc = np.ascontiguousarray(form.facets, dtype=np.int32)
            self._facets = fc
            if form.kind in _lib.INTERIOR_FACET_KINDS:
                _lib.check(_lib.lib.fe_form_set_interior_facets(self._handle, fc.ctypes.data, len(fc)),
                           "fe_form_set_interior_facets")
            else:
                _lib.check(_lib.lib.fe_form_set_facets(self._handle, fc.ctypes.data, len(fc)), "fe_form_set_facets")
        if form.precision == "fp32":
            _lib.check(_lib.lib.fe_form_set_precision(self._handle, _lib.PREC_FP32), "fe_form_set_precision")
        self._bound_sparsity = None
        self._coef_refs: list = [None] * len(form.coefficients)
        nc = len(form.coefficients)
        self._coef_ring: list = [None] * nc   # per coefficient: COEF_RING device copies (large uploads)
        self._coef_slot: list = [0] * nc      # the copy the engine reads now
        self._coef_free: list = [[None] * COEF_RING for _ in range(nc)]  # per copy: event after its last tracked read
        self._external = getattr(self, "_external", False)
        self._aux_dofmaps: dict = {}
        self.to_device()

    # -- restriction (CUDAForm::set_restriction, cpp/cudolfinx/fem/CUDAForm.h:201-232) --
    def set_restriction(self, restrictions: typing.Sequence[typing.Optional[np.ndarray]]):
        """Restrict the form's spaces (one entry per argument, None = the whole
        space): cell dofs outside a restriction take no entries and the kept
        dofs are numbered by their position in it."""
        if len(restrictions) != self.rank:
            raise ValueError("Number of restrictions must equal arity of form (1 for vector, 2 for matrix)!")
        if self._part == "diagonal":  # one space: the test restriction is the trial one
            restrictions = [restrictions[0], restrictions[0]]
        old = [dm.restriction for dm in self._dofmaps]
        new = [None if r is None else np.ascontiguousarray(r, dtype=np.int32) for r in restrictions]
        if all((o is None and n is None) or (o is not None and n is not None and np.array_equal(o, n))
               for o, n in zip(old, new)):
            return
        self._dofmaps = [device_dofmap(self._ctx, V) if r is None else DeviceDofMap(self._ctx, V, r)
                         for V, r in zip(self._spec.function_spaces, new)]
        self._create_handle()

    def restriction(self, i: int):
        """Restriction of argument i (None: the whole space)."""
        return self._dofmaps[i].restriction

    def space_size(self, i: int) -> int:
        """Scalar size of argument i's (restricted) space."""
        return self._dofmaps[i].size

    # -- coefficients -------------------------------------------------------
    def _set_coefficient(self, i: int, c):
        ctx = self._ctx
        ncomp = 3 if self._spec.kind in ("VP2_LOAD", "VP2_FACET_LOAD") else 1
        C = self._spec.mesh.num_cells
        if isinstance(c, Function):
            V = c.function_space
            vals = np.ascontiguousarray(c.x.array, dtype=np.float64)
            if V.family == "DG" and V.degree == 0:
                kind, cmap = _lib.COEFF_DG0, None
            elif V.family == "DG" and V.degree == 1:
                # vertex values through the DG1 dofmap: the engine's 4-dof
                # vertex-field coefficient (FE_COEFF_P1)
                kind, cmap = _lib.COEFF_P1, device_dofmap(ctx, V)
                self._aux_dofmaps[i] = cmap
            elif V.degree == 1 and V.bs == 1:
                kind, cmap = _lib.COEFF_P1, device_dofmap(ctx, V)
                self._aux_dofmaps[i] = cmap
            elif V.degree == 2 and V.bs == 1 and self._spec.kind == "P2_ENERGY":
                kind, cmap = _lib.COEFF_P2, device_dofmap(ctx, V)
                self._aux_dofmaps[i] = cmap
            else:
                raise ValueError("coefficients must be constants, DG0 or scalar P1 Functions")
            self._coef_refs[i] = vals
            return self._upload(i, kind, cmap.handle if cmap else None, vals)
        if hasattr(c, "data_ptr"):  # device tensor: DG0 values read in place
            if c.numel() != C * ncomp:
                raise ValueError("device coefficient arrays must hold one value per cell (DG0)")
            self._coef_refs[i] = c
            _lib.check(_lib.lib.fe_form_set_coefficient(self._handle, i, _lib.COEFF_DG0, None, c.data_ptr(),
                                                        c.numel(), 1, ctx.stream()), "fe_form_set_coefficient")
            return None
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
        if kind == _lib.COEFF_CONSTANT:
            _lib.check(_lib.lib.fe_form_set_coefficient(self._handle, i, kind, None, arr.ctypes.data, arr.size, 0,
                                                        ctx.stream()), "fe_form_set_coefficient")
            return None
        return self._upload(i, kind, None, arr)

    def _upload(self, i: int, kind: int, cmap, arr: np.ndarray):
        """Host -> device copy of coefficient i on the context's upload stream,
        into the next of the coefficient's COEF_RING device copies, which the
        engine then reads in place.  The copy waits only for the last tracked
        kernels that read that device copy (so it overlaps the kernels still
        reading the newer copies, on any stream), or for all work queued on
        the current stream when that is unknown."""
        ctx = self._ctx
        if arr.nbytes < OVERLAP_MIN_BYTES:
            # small copies: the event round trip would cost more than the overlap
            _lib.check(_lib.lib.fe_form_set_coefficient(self._handle, i, kind, cmap, arr.ctypes.data, arr.size, 0,
                                                        ctx.stream()), "fe_form_set_coefficient")
            return None
        self._overlapped = True
        up = ctx.upload_stream()
        ring = self._coef_ring[i]
        if ring is None or ring[0].numel() != arr.size:
            # (the old copies carry record_stream marks of their uploads and
            # readers: the allocator reuses them only after those finish)
            ring = [torch.empty(arr.size, dtype=torch.float64, device=ctx.torch_device) for _ in range(COEF_RING)]
            self._coef_ring[i] = ring
            self._coef_free[i] = [None] * COEF_RING
        slot = (self._coef_slot[i] + 1) % COEF_RING
        free = self._coef_free[i][slot]
        if self._external or free is None:
            up.wait_stream(ctx.torch_stream())
        else:
            up.wait_event(free)
        with torch.cuda.stream(up):
            ring[slot].copy_(torch.from_numpy(arr), non_blocking=True)
        ring[slot].record_stream(up)
        _lib.check(_lib.lib.fe_form_set_coefficient(self._handle, i, kind, cmap, ring[slot].data_ptr(), arr.size, 1,
                                                    up.cuda_stream), "fe_form_set_coefficient")
        self._coef_slot[i] = slot
        ev = torch.cuda.Event()
        ev.record(up)
        return ev

    def to_device(self, coefficients: typing.Optional[list] = None):
        """Copy host-side coefficient values to the device (CUDAForm.h:195-199).
        With ``coefficients`` given, only those Functions are re-uploaded.  The
        copies run on the context's upload stream; work enqueued afterwards on
        the current stream waits for them."""
        cur = self._ctx.torch_stream()
        for i, c in enumerate(self._spec.coefficients):
            if coefficients is None or any(c is q for q in coefficients):
                ev = self._set_coefficient(i, c)
                if ev is not None:
                    cur.wait_event(ev)

    def _mark_used(self):
        """Record that the kernels enqueued so far on the current stream read
        this form's coefficient buffers (the next upload into them waits).
        Only forms with side-stream uploads need it."""
        if not getattr(self, "_overlapped", False):
            return
        cur = self._ctx.torch_stream()
        ev = torch.cuda.Event()
        ev.record(cur)
        for i in range(len(self._coef_free)):
            self._coef_free[i][self._coef_slot[i]] = ev
            if self._coef_ring[i] is not None:
                self._coef_ring[i][self._coef_slot[i]].record_stream(cur)

    # -- pattern binding ----------------------------------------------------
    def _bind(self, sparsity):
        if self._bound_sparsity is not sparsity:
            _lib.check(_lib.lib.fe_form_bind_sparsity(self._handle, sparsity.handle, self._ctx.stream()),
                       "fe_form_bind_sparsity")
            self._bound_sparsity = sparsity

    def _bind_block(self, sparsity, row_offset: int, col_offset: int):
        """Bind as block (i, j) of a monolithic pattern at scalar offsets."""
        key = (row_offset, col_offset)
        if self._bound_sparsity is not sparsity or getattr(self, "_block_offsets", None) != key:
            _lib.check(_lib.lib.fe_form_bind_sparsity_block(self._handle, sparsity.handle, int(row_offset),
                                                            int(col_offset), self._ctx.stream()),
                       "fe_form_bind_sparsity_block")
            self._bound_sparsity = sparsity
            self._block_offsets = key

    def _integral_handles(self) -> list:
        """Engine forms whose sum is this form (one per integral)."""
        return [self._handle]

    def _needs_union_pattern(self) -> bool:
        """Whether the matrix pattern must join the two cells of interior facets."""
        return self._spec.kind in _lib.INTERIOR_FACET_KINDS

    # -- properties mirroring the reference --------------------------------
    @property
    def cuda_form(self):
        """The engine form handle, for direct C-ABI calls.  Once handed out,
        coefficient uploads wait for everything queued on the current stream
        (kernels launched through the handle are not tracked)."""
        self._external = True
        return self._handle

    @property
    def cuda_mesh(self):
        return self._cuda_mesh

    @property
    def dolfinx_form(self) -> FormSpec:
        return self._spec

    @property
    def function_spaces(self):
        return self._spec.function_spaces[:self.rank]

    @property
    def rank(self) -> int:
        return 1 if self._part == "diagonal" else self._spec.rank

    @property
    def part(self) -> str:
        """'full', or 'diagonal' for the diagonal of a bilinear form."""
        return self._part

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h:
            self._handle = None
            release = getattr(_lib, "release", None)  # None during interpreter teardown
            if release is not None:
                release("fe_form_destroy", h)


class FFCxCUDAForm(CUDAForm):
    """CUDA wrapper of a form given as FFCx tabulate_tensor bodies, the
    reference's general path (python/cudolfinx/form.py:26-105: the form's
    integrals wrapped by jit.py and compiled with NVRTC).  One engine form per
    integral (fe_form_create_ffcx), all on the same spaces, coefficients and
    constants; assembling the form sums its integrals.  ``cachedir`` keeps the
    compiled kernels on disk (the reference's cudolfinx cache directory)."""

    def __init__(self, form: FFCxForm, jit_args: typing.Optional[dict] = None, cachedir: typing.Optional[str] = None):
        if not isinstance(form, FFCxForm):
            raise TypeError(f"Expected a cudolfinx.fem.FFCxForm, got '{type(form)}'")
        if not form.integrals:
            raise ValueError("a form needs at least one integral")
        if form.rank > 2:
            raise ValueError("forms of rank above 2 are not supported")
        self._ctx = get_cuda_context()
        self._spec = form
        self._part = "full"
        self._cachedir = cachedir
        self._cuda_mesh = _create_mesh_on_device(self._ctx, form.mesh)
        self._dofmaps = [device_dofmap(self._ctx, V) for V in form.function_spaces]
        self._coef_maps = [device_dofmap(self._ctx, c.function_space) for c in form.coefficients]
        self._jit_args = dict(DEFAULT_CUDA_JIT_ARGS, **(jit_args or {}))
        self._handles = []
        self._handle = None
        self._create_handle()

    def _create_handle(self):
        from . import fem as _fem

        self._destroy_handles()
        form = self._spec
        given = [c.function_space.dofs_per_cell * c.function_space.bs for c in form.coefficients]
        if form.coefficient_sizes is not None:
            if len(form.coefficient_sizes) != len(given):
                raise RuntimeError(f"the form has {len(form.coefficient_sizes)} coefficient(s), "
                                   f"{len(given)} given")
            for q, (want, got) in enumerate(zip(form.coefficient_sizes, given)):
                if int(want) != got:
                    raise RuntimeError(f"coefficient {q} has {int(want)} values per cell in the compiled form; "
                                       f"its function space gives {got}")
        sizes = (ctypes.c_int * max(1, len(given)))(*given)
        test = self._dofmaps[0].handle if form.rank >= 1 else None
        trial = self._dofmaps[1].handle if form.rank == 2 else None
        consts = form.packed_constants()
        self._entities = []
        for itg in form.integrals:
            if itg.integral_type not in _lib.INTEGRAL:
                raise ValueError(f"unknown integral type {itg.integral_type!r}")
            h = _lib.out_handle()
            _lib.check(_lib.lib.fe_form_create_ffcx(
                self._ctx.handle, self._cuda_mesh.handle, test, trial, _lib.INTEGRAL[itg.integral_type],
                itg.name.encode(), itg.body.encode(), len(form.coefficients), sizes, len(consts),
                self._cachedir.encode() if self._cachedir else None, h), "fe_form_create_ffcx")
            self._handles.append(h.value)
            if itg.integral_type == "exterior_facet":
                ent = itg.entities if itg.entities is not None else _fem.exterior_facets(form.mesh)
                ent = np.ascontiguousarray(ent, dtype=np.int32)
                _lib.check(_lib.lib.fe_form_set_facets(h.value, ent.ctypes.data, len(ent)), "fe_form_set_facets")
                self._entities.append(ent)
            elif itg.integral_type == "interior_facet":
                ent = itg.entities if itg.entities is not None else _fem.interior_facets(form.mesh)
                ent = np.ascontiguousarray(ent, dtype=np.int32)
                _lib.check(_lib.lib.fe_form_set_interior_facets(h.value, ent.ctypes.data, len(ent)),
                           "fe_form_set_interior_facets")
                self._entities.append(ent)
        self._handle = self._handles[0]
        self._bound_sparsity = None
        self._external = getattr(self, "_external", False)
        self._coef_dev = [None] * len(form.coefficients)
        self.to_device()

    def _destroy_handles(self):
        for h in getattr(self, "_handles", []):
            _lib.lib.fe_form_destroy(h)
        self._handles = []
        self._handle = None

    def set_restriction(self, restrictions):
        if len(restrictions) != self.rank:
            raise ValueError("Number of restrictions must equal arity of form (1 for vector, 2 for matrix)!")
        new = [None if r is None else np.ascontiguousarray(r, dtype=np.int32) for r in restrictions]
        old = [dm.restriction for dm in self._dofmaps]
        if all((o is None and n is None) or (o is not None and n is not None and np.array_equal(o, n))
               for o, n in zip(old, new)):
            return
        self._dofmaps = [device_dofmap(self._ctx, V) if r is None else DeviceDofMap(self._ctx, V, r)
                         for V, r in zip(self._spec.function_spaces, new)]
        self._create_handle()

    def to_device(self, coefficients: typing.Optional[list] = None):
        """Copy the coefficients' host values and the constants to the device
        (the reference re-uploads them on every assembly call,
        assemble.py:100-103); every integral reads the same device arrays."""
        ctx = self._ctx
        for q, c in enumerate(self._spec.coefficients):
            if coefficients is not None and not any(c is x for x in coefficients):
                continue
            V = c.function_space
            vals = c.x.array
            if hasattr(vals, "data_ptr"):  # a device tensor: read in place
                dev = vals
            else:
                host = torch.from_numpy(np.ascontiguousarray(vals, dtype=np.float64))
                dev = self._coef_dev[q]
                if dev is None or dev.numel() != host.numel():
                    dev = torch.empty(host.numel(), dtype=torch.float64, device=ctx.torch_device)
                dev.copy_(host)
            self._coef_dev[q] = dev
            for h in self._handles:
                _lib.check(_lib.lib.fe_form_set_coefficient_field(h, q, self._coef_maps[q].handle, dev.data_ptr(),
                                                                  V.num_nodes * V.bs, 1, ctx.stream()),
                           "fe_form_set_coefficient_field")
        consts = np.ascontiguousarray(self._spec.packed_constants())
        self._consts = consts
        for h in self._handles:
            _lib.check(_lib.lib.fe_form_set_constants(h, consts.ctypes.data if consts.size else None, consts.size,
                                                      ctx.stream()), "fe_form_set_constants")

    def _bind(self, sparsity):
        if self._bound_sparsity is not sparsity:
            for h in self._handles:
                _lib.check(_lib.lib.fe_form_bind_sparsity(h, sparsity.handle, self._ctx.stream()),
                           "fe_form_bind_sparsity")
            self._bound_sparsity = sparsity

    def _bind_block(self, sparsity, row_offset: int, col_offset: int):
        key = (row_offset, col_offset)
        if self._bound_sparsity is not sparsity or getattr(self, "_block_offsets", None) != key:
            for h in self._handles:
                _lib.check(_lib.lib.fe_form_bind_sparsity_block(h, sparsity.handle, int(row_offset), int(col_offset),
                                                                self._ctx.stream()), "fe_form_bind_sparsity_block")
            self._bound_sparsity = sparsity
            self._block_offsets = key

    def _integral_handles(self) -> list:
        return list(self._handles)

    def _needs_union_pattern(self) -> bool:
        return any(i.integral_type == "interior_facet" for i in self._spec.integrals)

    def __del__(self):
        hs = getattr(self, "_handles", None)
        if hs:
            self._handles = []
            self._handle = None
            release = getattr(_lib, "release", None)  # None during interpreter teardown
            if release is not None:
                for h in hs:
                    release("fe_form_destroy", h)


class BlockCUDAForm:
    """Forms of a block system (mirrors python/cudolfinx/form.py:107-225).

    A list of linear forms is a block vector; a list of lists of bilinear
    forms (None for an empty block) is a block matrix.  Block i occupies the
    scalar range [offsets[i], offsets[i+1]) of the monolithic vector / matrix,
    its size that of its (restricted) space.  ``restrictions``: for a vector
    one array (or None) per form; for a matrix a pair (row restrictions,
    column restrictions).  Each array lists the kept block dofs of the space,
    sorted; kept dofs are numbered by their position in it."""

    def __init__(self, forms, restrictions=None):
        self._forms = forms
        self._restrictions = restrictions
        if not len(forms):
            raise ValueError("Must provide at least one form!")
        if isinstance(forms[0], CUDAForm):
            self._init_vector()
        else:
            self._init_matrix()

    @staticmethod
    def _offsets(sizes):
        off = [0]
        for n in sizes:
            off.append(off[-1] + n)
        return off

    def _init_vector(self):
        for i, f in enumerate(self._forms):
            if f.rank != 1:
                raise ValueError("a block vector takes linear forms")
            r = None if self._restrictions is None else self._restrictions[i]
            f.set_restriction([r])
        self._offsets_list = self._offsets([f.space_size(0) for f in self._forms])
        self._row_offsets = self._col_offsets = self._offsets_list

    def _init_matrix(self):
        rows, cols = len(self._forms), len(self._forms[0])
        if any(len(r) != cols for r in self._forms):
            raise ValueError("a block matrix needs rows of equal length")
        rr = [None] * rows if self._restrictions is None else list(self._restrictions[0])
        cr = [None] * cols if self._restrictions is None else list(self._restrictions[1])
        if len(rr) != rows or len(cr) != cols:
            raise ValueError("one restriction per block row and per block column")
        rsize, csize = [None] * rows, [None] * cols
        for i, row in enumerate(self._forms):
            for j, f in enumerate(row):
                if f is None:
                    continue
                if f.rank != 2:
                    raise ValueError("a block matrix takes bilinear forms")
                f.set_restriction([rr[i], cr[j]])
                for sizes, k, idx in ((rsize, 0, i), (csize, 1, j)):
                    n = f.space_size(k)
                    if sizes[idx] is not None and sizes[idx] != n:
                        raise ValueError("the forms of a block row / column act on spaces of different sizes")
                    sizes[idx] = n
        if any(n is None for n in rsize) or any(n is None for n in csize):
            raise ValueError("every block row and column needs at least one form")
        self._row_offsets = self._offsets(rsize)
        self._col_offsets = self._offsets(csize)
        self._offsets_list = self._row_offsets

    @property
    def forms(self):
        """Return the list of forms."""
        return self._forms

    @property
    def dolfinx_forms(self):
        return [f.dolfinx_form if isinstance(f, CUDAForm) else [g.dolfinx_form if g else None for g in f]
                for f in self._forms]

    @property
    def offsets(self):
        """Scalar offsets of the blocks (rows for a block matrix)."""
        return self._offsets_list

    @property
    def row_offsets(self):
        return self._row_offsets

    @property
    def col_offsets(self):
        return self._col_offsets

    @property
    def local_size(self):
        """Size of the monolithic vector (rows of the block matrix)."""
        return self._offsets_list[-1]

    @property
    def global_size(self):
        return self.local_size


def form(form: typing.Union[FormSpec, typing.Iterable], restriction=None,
         cuda_jit_args: typing.Optional[dict] = None, **kwargs):
    """Create a CUDAForm from a built-in form spec, or a BlockCUDAForm from a
    list of them (block vector) or a list of lists (block matrix, None for an
    empty block) with optional restrictions (mirrors cudolfinx.form,
    python/cudolfinx/form.py:227-249).  Of the keyword arguments the reference
    forwards to dolfinx.fem.form, ``form_compiler_options={"part": "diagonal"}``
    is honoured: the bilinear form's diagonal becomes a linear form."""
    fco = kwargs.get("form_compiler_options") or {}
    part = fco.get("part")
    cachedir = kwargs.get("cachedir")
    if isinstance(form, FFCxForm):
        if part not in (None, "full"):
            raise ValueError("the diagonal of a form given as FFCx bodies is compiled by FFCx as a linear form")
        f = FFCxCUDAForm(form, cuda_jit_args, cachedir)
        if restriction is not None:
            f.set_restriction(restriction)
        return f
    if isinstance(form, FormSpec):
        f = CUDAForm(form, cuda_jit_args, part)
        if restriction is not None:
            f.set_restriction(restriction)
        return f

    def _create(x):
        if x is None:
            return None
        if isinstance(x, FFCxForm):
            return FFCxCUDAForm(x, cuda_jit_args, cachedir)
        if isinstance(x, FormSpec):
            return CUDAForm(x, cuda_jit_args, part)
        return [_create(y) for y in x]

    return BlockCUDAForm(_create(form), restriction)
