"""Collections of Dirichlet BCs on the device (mirrors python/cudolfinx/bcs.py:12-79).

As in the reference, BCs are grouped by function space and each group becomes
one device object holding per-dof markers, the BC dof list (owned first; on
one GPU every dof is owned) and a full-length value array g
(cpp/cudolfinx/fem/CUDADirichletBC.h:56-194).
"""
from __future__ import annotations

import typing

import numpy as np

from . import _lib
from .fem import DirichletBC, FunctionSpace


class _DeviceBC:
    def __init__(self, ctx, V: FunctionSpace, bcs: list[DirichletBC]):
        self.ctx = ctx
        self.V = V
        n = V.num_dofs
        markers = np.zeros(n, dtype=np.uint8)
        g = np.zeros(n)
        dofs = []
        for bc in bcs:
            markers[bc.dofs] = 1
            vals = bc.values()
            g[bc.dofs] = vals[bc.dofs]
            dofs.append(bc.dofs)
        d = np.unique(np.concatenate(dofs)).astype(np.int32) if dofs else np.zeros(0, dtype=np.int32)
        self.dofs = np.ascontiguousarray(d)
        self.g = np.ascontiguousarray(g)
        self.markers = markers
        h = _lib.out_handle()
        _lib.check(_lib.lib.fe_bc_create(ctx.handle, n, markers.ctypes.data,
                                         self.dofs.ctypes.data if len(self.dofs) else None,
                                         len(self.dofs), len(self.dofs), self.g.ctypes.data, h), "fe_bc_create")
        self.handle = h.value
        self.bcs = list(bcs)

    def update(self, bcs: list[DirichletBC]):
        for bc in bcs:
            vals = bc.values()
            self.g[bc.dofs] = vals[bc.dofs]
        _lib.check(_lib.lib.fe_bc_update(self.handle, self.g.ctypes.data, self.ctx.stream()), "fe_bc_update")
        for r in getattr(self, "_restricted", {}).values():
            r.refresh()

    def restricted(self, restriction: np.ndarray) -> "_RestrictedBC":
        """The same BCs in the numbering of a restricted space (kept block
        dofs `restriction`, sorted): BC dofs outside it are dropped."""
        if not hasattr(self, "_restricted"):
            self._restricted = {}
            self._by_id = {}
        # a form hands out the same restriction array on every call: look it up
        # by identity first, by content (hashing the whole array) only once
        hit = self._by_id.get(id(restriction))
        if hit is not None and hit[0] is restriction:
            return hit[1]
        key = np.ascontiguousarray(restriction, dtype=np.int32).tobytes()
        r = self._restricted.get(key)
        if r is None:
            r = _RestrictedBC(self, np.frombuffer(key, dtype=np.int32))
            self._restricted[key] = r
        self._by_id[id(restriction)] = (restriction, r)
        return r

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self.handle = None
            release = getattr(_lib, "release", None)  # None during interpreter teardown
            if release is not None:
                release("fe_bc_destroy", h)


class _RestrictedBC:
    """Device BC object of a restricted space, derived from a _DeviceBC."""

    def __init__(self, parent: _DeviceBC, restriction: np.ndarray):
        self.parent = parent
        bs = parent.V.bs
        self.kept = (restriction.astype(np.int64)[:, None] * bs + np.arange(bs)).ravel()
        self.markers = np.ascontiguousarray(parent.markers[self.kept])
        self.dofs = np.ascontiguousarray(np.nonzero(self.markers)[0].astype(np.int32))
        self.g = np.ascontiguousarray(parent.g[self.kept])
        h = _lib.out_handle()
        n = len(self.kept)
        _lib.check(_lib.lib.fe_bc_create(parent.ctx.handle, n, self.markers.ctypes.data,
                                         self.dofs.ctypes.data if len(self.dofs) else None, len(self.dofs),
                                         len(self.dofs), self.g.ctypes.data, h), "fe_bc_create")
        self.handle = h.value

    def refresh(self):
        self.g[:] = self.parent.g[self.kept]
        _lib.check(_lib.lib.fe_bc_update(self.handle, self.g.ctypes.data, self.parent.ctx.stream()), "fe_bc_update")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self.handle = None
            release = getattr(_lib, "release", None)  # None during interpreter teardown
            if release is not None:
                release("fe_bc_destroy", h)


class CUDADirichletBC:
    """Represents a collection of boundary conditions."""

    def __init__(self, ctx, bcs: typing.List[DirichletBC]):
        self.bcs = list(bcs)
        self._ctx = ctx
        self._function_spaces: list[FunctionSpace] = []
        self._bc_lists: list[list[DirichletBC]] = []
        for bc in self.bcs:
            V = bc.function_space
            for i, W in enumerate(self._function_spaces):
                if W is V:
                    self._bc_lists[i].append(bc)
                    break
            else:
                self._function_spaces.append(V)
                self._bc_lists.append([bc])
        self._device_bcs = [_DeviceBC(ctx, V, L) for V, L in zip(self._function_spaces, self._bc_lists)]

    def _get_cpp_bcs(self, V: FunctionSpace, restriction: typing.Optional[np.ndarray] = None):
        """Device BC object for V (in the numbering of `restriction` when
        given), or None (no BCs on V) like the reference's empty collection."""
        for W, d in zip(self._function_spaces, self._device_bcs):
            if W is V:
                return d if restriction is None else d.restricted(restriction)
        return None

    def update(self, bcs: typing.Optional[typing.List[DirichletBC]] = None):
        """Re-upload BC values (time-dependent BCs); by default all of them."""
        bcs = self.bcs if bcs is None else bcs
        for V, d in zip(self._function_spaces, self._device_bcs):
            d.update([bc for bc in bcs if bc.function_space is V])
