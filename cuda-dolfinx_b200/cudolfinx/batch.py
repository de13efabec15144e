"""Many independent assemblies in one CUDA graph, with a variant autotuner.

No counterpart in the reference, which launches one assembly per Python call
with a context synchronisation after every kernel (cpp/cudolfinx/fem/
CUDAFormIntegral.cpp:2354-2361).  Here a list of (form, matrix, BCs) items --
meshes of different sizes, P1 and P2 forms mixed -- is assembled through the
C-ABI on one stream, captured once into a CUDA graph and replayed with a
single launch call.  ``VariantTuner`` times the matrix variants that apply to
each (form kind, precision, size class) on the device and keeps the fastest;
the graph is captured with the chosen variant per item.
"""
from __future__ import annotations

import math
import typing

import torch

from . import _lib
from .bcs import CUDADirichletBC
from .context import get_cuda_context
from .form import CUDAForm
from .la import CUDAMatrix

# matrix variants worth timing per form kind (all parity-tested)
CANDIDATES = {
    "P1_STIFFNESS": ("atomic", "block", "tile"),
    "P2_STIFFNESS": ("atomic", "block", "grouped", "coalesced"),
    "VP2_ELASTICITY": ("coalesced", "atomic", "atomic-full"),
    "P3_STIFFNESS": ("coalesced", "atomic"),  # coalesced: FP64 element tensors only (skipped for FP32)
}
# launch shapes of the atomic scatter timed per form kind: (cells per CTA,
# byte maps staged in shared memory)
LAUNCHES = {
    "P1_STIFFNESS": ((128, 1), (64, 1), (32, 1)),
    "P2_STIFFNESS": ((128, 1), (64, 1), (32, 1), (128, 0), (64, 0)),
}


class VariantTuner:
    """Chooses the fastest matrix variant per (form kind, precision, size
    class) and, for the atomic scatter, its launch shape (cells per CTA and
    shared-memory staging of the byte maps); size classes are powers of two of
    the cell count.  ``choose`` returns the variant name and leaves the
    chosen launch shape set on the form."""

    def __init__(self, reps: int = 3):
        self.reps = reps
        self.cache: dict = {}
        self.timings: dict = {}

    @staticmethod
    def key(a: CUDAForm) -> tuple:
        C = a._spec.mesh.num_cells
        coef = tuple(type(c).__name__ + (str(c.function_space.degree) if hasattr(c, "function_space") else "")
                     for c in a._spec.coefficients)
        return (a._spec.kind, a._spec.precision, coef, int(math.log2(max(1, C))))

    def choose(self, a: CUDAForm, mat: CUDAMatrix, bc0, bc1) -> str:
        k = self.key(a)
        if k in self.cache:
            v, shape = self.cache[k]
            _lib.check(_lib.lib.fe_form_set_launch(a.cuda_form, *shape), "fe_form_set_launch")
            return v
        stream = torch.cuda.current_stream()
        sp = stream.cuda_stream
        best, best_ms, times = None, float("inf"), {}
        trials = []
        for v in CANDIDATES.get(a._spec.kind, ("atomic",)):
            shapes = LAUNCHES.get(a._spec.kind, ((0, 1),)) if v in ("atomic", "atomic-full") else ((0, 1),)
            trials += [(v, shape) for shape in shapes]
        for v, shape in trials:
            flags = _lib.ASM_ZERO | _lib.VARIANT_FLAGS[v]
            _lib.check(_lib.lib.fe_form_set_launch(a.cuda_form, *shape), "fe_form_set_launch")

            def call():
                _lib.check(_lib.lib.fe_assemble_matrix(a.cuda_form, mat.values.data_ptr(), bc0, bc1, 1.0, flags, sp),
                           "fe_assemble_matrix")

            try:
                call()  # plan build
            except RuntimeError:
                continue  # variant not offered for this form (e.g. a P1 coefficient in the block kernel)
            call()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(self.reps):
                call()
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / self.reps
            times[(v,) + tuple(shape)] = ms
            if ms < best_ms:
                best, best_ms = (v, tuple(shape)), ms
        if best is None:
            best = ("atomic", (0, 1))
        _lib.check(_lib.lib.fe_form_set_launch(a.cuda_form, *best[1]), "fe_form_set_launch")
        self.cache[k] = best
        self.timings[k] = times
        return best[0]


class AssemblyGraph:
    """Matrix assemblies of many (form, matrix, BCs) items captured into one
    CUDA graph.  ``variants``: "auto" (engine default per item), "tune" (a
    VariantTuner picks per item) or one variant name for every item.
    ``branches``: independent streams the capture spreads the items over (a
    graph with that many parallel branches, balanced by nonzeros; items of
    one form stay on one branch), so that the launches of small meshes
    overlap (64 meshes, n = 8..64, on B200: 8.70 ms per replay with 8
    branches, 8.77 with 4, 9.48 with 1)."""

    def __init__(self, items: typing.Sequence[tuple], variants: str = "tune",
                 tuner: typing.Optional[VariantTuner] = None, branches: int = 8):
        self._ctx = get_cuda_context()
        self.branches = max(1, int(branches))
        self.items = []
        for a, mat, bcs in items:
            if not isinstance(a, CUDAForm) or a.rank != 2:
                raise TypeError("items must hold bilinear CUDAForms")
            a._bind(mat.sparsity)
            col = bcs if isinstance(bcs, CUDADirichletBC) or bcs is None else CUDADirichletBC(self._ctx, list(bcs))
            bc0 = col._get_cpp_bcs(a.function_spaces[0]) if col else None
            bc1 = col._get_cpp_bcs(a.function_spaces[1]) if col else None
            self.items.append({"a": a, "mat": mat, "col": col, "bc0": bc0.handle if bc0 else None,
                               "bc1": bc1.handle if bc1 else None})
        self.tuner = tuner or VariantTuner()
        for it in self.items:
            if variants == "tune":
                it["variant"] = self.tuner.choose(it["a"], it["mat"], it["bc0"], it["bc1"])
            else:
                it["variant"] = variants
        self.graph = None
        self._stream = None

    def _launch_all(self, sp, items=None):
        for it in self.items if items is None else items:
            flags = _lib.ASM_ZERO | _lib.VARIANT_FLAGS[it["variant"]]
            _lib.check(_lib.lib.fe_assemble_matrix(it["a"].cuda_form, it["mat"].values.data_ptr(), it["bc0"],
                                                   it["bc1"], 1.0, flags, sp), "fe_assemble_matrix")

    def _branch_items(self, nb: int) -> list:
        """Items spread over nb branches: the forms' item lists, largest
        first, each onto the branch with the fewest nonzeros so far."""
        by_form: dict = {}
        for it in self.items:
            by_form.setdefault(id(it["a"]), []).append(it)
        lists = sorted(by_form.values(), key=lambda L: -sum(it["mat"].sparsity.nnz for it in L))
        out = [[] for _ in range(nb)]
        load = [0] * nb
        for L in lists:
            b = load.index(min(load))
            out[b] += L
            load[b] += sum(it["mat"].sparsity.nnz for it in L)
        return [o for o in out if o]

    def run_eager(self):
        """The same launches without the graph (one C-ABI call per item)."""
        self._launch_all(torch.cuda.current_stream().cuda_stream)

    def capture(self):
        # plans and caches are built outside the capture
        self.run_eager()
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        self._stream = torch.cuda.Stream()
        groups = self._branch_items(self.branches)
        self._branch_streams = [torch.cuda.Stream() for _ in groups[1:]]
        with torch.cuda.graph(self.graph, stream=self._stream):
            cap = torch.cuda.current_stream()
            for st in self._branch_streams:  # fork
                st.wait_stream(cap)
            self._launch_all(cap.cuda_stream, groups[0] if groups else [])
            for st, g in zip(self._branch_streams, groups[1:]):
                self._launch_all(st.cuda_stream, g)
            for st in self._branch_streams:  # join
                cap.wait_stream(st)
        torch.cuda.synchronize()
        return self

    def replay(self):
        if self.graph is None:
            raise RuntimeError("capture() first")
        self.graph.replay()

    @property
    def nnz(self) -> int:
        return sum(it["mat"].sparsity.nnz for it in self.items)
