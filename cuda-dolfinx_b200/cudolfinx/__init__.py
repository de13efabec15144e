"""cudolfinx API on the B200-native assembly engine (libcudolfinx_b200.so).

Drop-in mirror of the reference's Python surface for the assembly path
(python/cudolfinx/__init__.py): ``form``, ``CUDAAssembler`` and the
``CUDAMatrix`` / ``CUDAVector`` / ``CUDADirichletBC`` handles.  ``fem`` holds
the host-side stand-ins for the DOLFINx objects those calls consume.
"""
from . import _lib, fem
from .assemble import CUDAAssembler
from .batch import AssemblyGraph, VariantTuner
from .bcs import CUDADirichletBC
from .context import get_cuda_context
from .form import CUDAForm, form
from .la import CUDAMatrix, CUDAVector, Sparsity

__all__ = ["AssemblyGraph", "CUDAAssembler", "CUDADirichletBC", "CUDAForm", "CUDAMatrix", "CUDAVector", "Sparsity", "fem", "form",
           "get_cuda_context", "VariantTuner"]
