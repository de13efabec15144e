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
from .coefficient import Coefficient
from .context import get_cuda_context
from .form import BlockCUDAForm, CUDAForm, FFCxCUDAForm, form
from .la import CUDAMatrix, CUDAVector, Sparsity



def release_caches(mesh=None):
    """Drop the module-level device caches (meshes, dofmaps, CSR patterns):
    all of them, or those of `mesh`.  Long-running processes that create many
    meshes call this to return device memory."""
    from .assemble import release_sparsity_cache
    from .form import release_device_caches
    release_sparsity_cache(mesh)
    release_device_caches(mesh)


__all__ = ["AssemblyGraph", "BlockCUDAForm", "FFCxCUDAForm", "CUDAAssembler", "CUDADirichletBC", "Coefficient", "CUDAForm", "CUDAMatrix", "CUDAVector", "Sparsity", "fem", "form",
           "get_cuda_context", "release_caches", "VariantTuner"]
