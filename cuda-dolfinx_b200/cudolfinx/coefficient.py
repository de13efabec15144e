"""Coefficient (mirrors python/cudolfinx/coefficient.py): a Function's value
vector on the device, with same-map interpolation from another Coefficient.

The reference wraps CUDACoefficient (cpp/cudolfinx/fem/CUDACoefficient.h:24-120):
a device copy of the dof vector, ``interpolate`` (the interpolation operator
of the two elements applied cell by cell on the device, then the result
copied back to the host) and ``values`` (the host copy).  Here the matrix
comes from ``fem.interpolation_matrix`` and the device work is
``fe_interpolate`` (one owner cell per target dof).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .context import get_cuda_context
from .fem import Function, interpolation_matrix
from .form import device_dofmap


class Coefficient:
    """CUDA wrapper of a Function: its dof vector on the device."""

    def __init__(self, f: Function):
        self._ctx = get_cuda_context()
        self._f = f
        self._V = f.function_space
        self._dofmap = device_dofmap(self._ctx, self._V)
        self._values = np.array(f.x.array, dtype=np.float64)
        self._d = torch.from_numpy(self._values).to(self._ctx.torch_device)

    def interpolate(self, coeff0: "Coefficient"):
        """Interpolate from another Coefficient on the same mesh, modifying this
        one's dof vector on the device and its host copy."""
        if not isinstance(coeff0, Coefficient):
            raise TypeError(f"Expected Coefficient, got '{type(coeff0)}'")
        if coeff0._V.mesh is not self._V.mesh:
            raise ValueError("interpolation between different meshes is not supported")
        im = interpolation_matrix(self._V, coeff0._V)
        _lib.check(_lib.lib.fe_interpolate(self._dofmap.handle, self._d.data_ptr(), coeff0._dofmap.handle,
                                           coeff0._d.data_ptr(), im.ctypes.data, self._ctx.stream()),
                   "fe_interpolate")
        torch.cuda.current_stream(self._ctx.device).synchronize()
        self._values[:] = self._d.cpu().numpy()

    def values(self) -> np.ndarray:
        """Return a copy of the dof vector (host)."""
        return self._values.copy()

    @property
    def device_values(self) -> torch.Tensor:
        return self._d
