"""ctypes binding of libcudolfinx_b200.so (the C ABI in include/cudolfinx_b200.h).

Plays the role of the reference's nanobind module ``cudolfinx.cpp``
(python/cudolfinx/wrappers/fem.cpp:74-407): every failing call raises
RuntimeError with the library's message, as nanobind does for the
reference's std::runtime_error.  There is no fallback: if the shared library
is missing or does not load, importing this module fails.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CUDOLFINX_B200_LIB",
                          os.path.join(os.path.dirname(_HERE), "lib", "libcudolfinx_b200.so"))

if not os.path.exists(LIB_PATH):
    raise ImportError(f"libcudolfinx_b200.so not found at {LIB_PATH}; build it with "
                      "`python cuda-dolfinx_b200/build.py`")

lib = ctypes.CDLL(LIB_PATH)

vp = ctypes.c_void_p
i64 = ctypes.c_int64
i32 = ctypes.c_int
u32 = ctypes.c_uint
dbl = ctypes.c_double
PP = ctypes.POINTER(ctypes.c_void_p)

FE_OK = 0
FE_ERR_NOT_CONVERGED = 6

# enum values (include/cudolfinx_b200.h)
FORM = {"P1_STIFFNESS": 1, "P2_STIFFNESS": 2, "VP2_ELASTICITY": 3, "P1_MASS": 9, "P2_MASS": 10, "VP2_MASS": 20, "P1_LOAD": 11, "P2_LOAD": 12, "VP2_LOAD": 13,
        "P1_FACET_MASS": 4, "P2_FACET_MASS": 5, "P1_FACET_LOAD": 14, "P2_FACET_LOAD": 15, "VP2_FACET_LOAD": 16,
        "INTEGRAL": 31, "P1_ENERGY": 32, "P2_ENERGY": 33, "FACET_INTEGRAL": 34,
        "P3_STIFFNESS": 6, "P3_LOAD": 17, "DG0_JUMP": 7, "DG1_JUMP": 8, "DG0_AVG_LOAD": 18, "DG1_AVG_LOAD": 19,
        "JUMP_NORM": 35}
INTERIOR_FACET_KINDS = ("DG0_JUMP", "DG1_JUMP", "DG0_AVG_LOAD", "DG1_AVG_LOAD", "JUMP_NORM")
COEFF_CONSTANT, COEFF_DG0, COEFF_P1, COEFF_P2 = 0, 1, 2, 3
INTEGRAL = {"cell": 0, "exterior_facet": 1, "interior_facet": 2}
PREC_FP64, PREC_FP32 = 0, 1
ASM_ZERO, ASM_DETERMINISTIC, ASM_ATOMIC, ASM_SORTED_SLOT, ASM_TILE, ASM_ROW_GATHER, ASM_BLOCK = 1, 2, 4, 8, 16, 32, 64
ASM_FULL_SCATTER = 128
ASM_GROUPED = 256
ASM_COALESCED = 512
VARIANT_FLAGS = {"auto": 0, "deterministic": ASM_DETERMINISTIC, "atomic": ASM_ATOMIC, "sorted-slot": ASM_SORTED_SLOT,
                 "tile": ASM_TILE, "row-gather": ASM_ROW_GATHER, "block": ASM_BLOCK, "atomic-full": ASM_ATOMIC | ASM_FULL_SCATTER, "grouped": ASM_GROUPED,
                 "coalesced": ASM_COALESCED}

_SIGS = {
    "fe_last_error": (ctypes.c_char_p, []),
    "fe_version": (ctypes.c_char_p, []),
    "fe_context_create": (i32, [i32, PP]),
    "fe_context_destroy": (i32, [vp]),
    "fe_context_synchronize": (i32, [vp]),
    "fe_mesh_create": (i32, [vp, vp, i64, vp, i64, i32, PP]),
    "fe_mesh_destroy": (i32, [vp]),
    "fe_dofmap_create": (i32, [vp, vp, i64, i32, i32, i64, PP]),
    "fe_dofmap_create_restricted": (i32, [vp, vp, i64, i32, i32, i64, PP]),
    "fe_dofmap_destroy": (i32, [vp]),
    "fe_sparsity_build": (i32, [vp, vp, PP]),
    "fe_sparsity_build_device": (i32, [vp, vp, vp, PP]),
    "fe_sparsity_build_block": (i32, [vp, i32, vp, vp, vp, vp, i64, i64, PP]),
    "fe_sparsity_build_forms": (i32, [i32, vp, PP]),
    "fe_sparsity_create": (i32, [vp, vp, vp, i64, i64, PP]),
    "fe_sparsity_info": (i32, [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64)]),
    "fe_sparsity_copy_to_host": (i32, [vp, vp, vp]),
    "fe_sparsity_device_arrays": (i32, [vp, PP, PP]),
    "fe_sparsity_destroy": (i32, [vp]),
    "fe_pattern_build_host": (i32, [vp, vp, i64, i32, i32, i32, i32, i64, i64, ctypes.POINTER(i64), PP, PP]),
    "fe_free_host": (None, [vp]),
    "fe_form_create": (i32, [vp, i32, vp, vp, vp, PP]),
    "fe_form_set_coefficient": (i32, [vp, i32, i32, vp, vp, i64, i32, vp]),
    "fe_form_set_precision": (i32, [vp, i32]),
    "fe_form_set_launch": (i32, [vp, i32, i32]),
    "fe_form_set_facets": (i32, [vp, vp, i64]),
    "fe_form_set_interior_facets": (i32, [vp, vp, i64]),
    "fe_assemble_scalar": (i32, [vp, ctypes.POINTER(dbl), vp]),
    "fe_form_bind_sparsity": (i32, [vp, vp, vp]),
    "fe_form_bind_sparsity_block": (i32, [vp, vp, i64, i64, vp]),
    "fe_form_destroy": (i32, [vp]),
    "fe_form_create_ffcx": (i32, [vp, vp, vp, vp, i32, ctypes.c_char_p, ctypes.c_char_p, i32, vp, i32,
                                  ctypes.c_char_p, PP]),
    "fe_form_set_coefficient_field": (i32, [vp, i32, vp, vp, i64, i32, vp]),
    "fe_form_set_constants": (i32, [vp, vp, i32, vp]),
    "fe_ffcx_source": (i32, [i32, i32, i32, i32, i32, i32, i32, vp, ctypes.c_char_p, ctypes.c_char_p, vp, i64,
                             ctypes.POINTER(i64)]),
    "fe_bc_create": (i32, [vp, i64, vp, vp, i64, i64, vp, PP]),
    "fe_bc_update": (i32, [vp, vp, vp]),
    "fe_bc_destroy": (i32, [vp]),
    "fe_assemble_matrix": (i32, [vp, vp, vp, vp, dbl, u32, vp]),
    "fe_assemble_matrix_batch": (i32, [vp, i32, vp, vp, vp, vp, dbl, u32, vp]),
    "fe_zero_entries": (i32, [vp, i64, vp]),
    "fe_assemble_diagonal": (i32, [vp, vp, u32, vp]),
    "fe_interpolate": (i32, [vp, vp, vp, vp, vp, vp]),
    "fe_assemble_vector": (i32, [vp, vp, u32, vp]),
    "fe_apply_lifting": (i32, [vp, i32, vp, vp, vp, dbl, vp]),
    "fe_set_bc": (i32, [vp, i64, vp, vp, dbl, vp]),
    "fe_assemble_rhs": (i32, [vp, vp, vp, vp, vp, dbl, u32, vp]),
    "fe_pcg_solve": (i32, [vp, vp, vp, vp, dbl, i32, ctypes.POINTER(i32), ctypes.POINTER(dbl), vp]),
    "fe_pcg_solve_noalloc": (i32, [vp, vp, vp, vp, dbl, i32, ctypes.POINTER(i32), ctypes.POINTER(dbl), vp]),
    "fe_pcg_solve_mixed": (i32, [vp, vp, vp, vp, dbl, dbl, i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32),
                                 ctypes.POINTER(dbl), vp]),
}

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = tuple(_SIGS)


def last_error() -> str:
    msg = lib.fe_last_error()
    return msg.decode() if msg else ""


def check(status: int, what: str = "") -> int:
    if status != FE_OK:
        raise RuntimeError(f"{what} failed (status {status}): {last_error()}")
    return status


def out_handle():
    return ctypes.c_void_p()


def release(destroy: str, handle) -> None:
    """Destroy an engine handle from a finalizer.  A no-op when the library
    object is already gone (interpreter shutdown clears module globals)."""
    L = globals().get("lib")
    if L is not None and handle:
        getattr(L, destroy)(handle)


def ptr(x) -> int | None:
    """Device/host address of a torch tensor, numpy array or int (None passes NULL)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(f"cannot take the address of {type(x)}")
