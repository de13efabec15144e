"""Assemble-and-solve request server on one GPU (continuous batching).

No counterpart in the reference: there a user script builds the mesh, forms
and matrix, assembles once and hands the objects to PETSc KSP
(examples/poisson.py:78-125), one problem per process.  This server accepts
requests as they arrive and keeps several of them on the device at once:

* a request names a problem family ("p1", "p2" Poisson or "vp2" elasticity)
  on the unit cube split into n^3 x 6 tets, carries its own DG0
  coefficients, and asks for the solution of A x = b with Dirichlet BCs to a
  relative residual ``rtol`` (on-device Jacobi-PCG);
* device state is cached per (family, n): the mesh, dofmaps and CSR pattern
  are shared, and "slots" (forms with their cell-to-slot maps, the matrix
  values, b, x and BC data) are reused by later requests with the same n;
* admission is by device-memory footprint: a request enters when a worker is
  free and its slot fits in the budget (idle slots of other sizes are evicted
  least-recently-used first); requests wait in arrival order otherwise, and a
  request larger than the whole budget is answered with an error;
* every worker drives its own CUDA stream, so the assemblies and solves of
  concurrent requests overlap on the device;
* vector-P2 solves run in mixed precision: inner Jacobi-PCG iterations on an
  FP32 copy of the matrix values in 3x3 blocks (4.4 instead of 12 bytes per
  nonzero), refined against the FP64 residual to the request's rtol; scalar
  P1 / P2 solves stay FP64 (their refinement restarts cost more iterations
  than the FP32 values save: P2 n=48 70.5 against 63.9 ms on B200).

``plain`` mode is the one-at-a-time FP64 path the server is compared with:
one worker, no caches (each request builds its mesh, pattern and forms),
FP64 element tensors, the FP64 solver.
"""
from __future__ import annotations

import collections
import dataclasses
import math
import threading
import time
import typing

import numpy as np

FAMILIES = ("p1", "p2", "vp2")


@dataclasses.dataclass
class Request:
    rid: int
    kind: str                        # "p1" | "p2" | "vp2"
    n: int                           # n^3 x 6 tets
    coef: typing.Tuple[np.ndarray, ...]  # DG0 per cell: (k,) or (lam, mu)
    arrival: float = 0.0             # seconds after the start of the run
    rtol: float = 1e-8

    @property
    def key(self) -> tuple:
        return (self.kind, self.n)


@dataclasses.dataclass
class Result:
    rid: int
    kind: str
    n: int
    x: typing.Optional[np.ndarray]
    iterations: int
    rel_residual: float
    arrival: float
    admitted: float
    done: float
    error: typing.Optional[str] = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


# ---------------------------------------------------------------------------
# sizes (exact for the unit-cube Kuhn meshes)
# ---------------------------------------------------------------------------
def problem_sizes(kind: str, n: int) -> dict:
    cells = 6 * n ** 3
    nv = (n + 1) ** 3
    edges = 3 * n * (n + 1) ** 2 + 3 * n * n * (n + 1) + n ** 3
    if kind == "p1":
        rows, nnz, k = nv, nv + 2 * edges, 4
    else:
        nodes = nv + edges
        nnz2 = 230 * n ** 3 + 138 * n ** 2 + 24 * n + 1
        rows, nnz, k = (nodes, nnz2, 10) if kind == "p2" else (3 * nodes, 9 * nnz2, 10)
    return {"cells": cells, "vertices": nv, "rows": rows, "nnz": nnz, "k": k}


def slot_bytes(kind: str, n: int) -> int:
    """Device bytes of one slot: CSR values, cell-to-slot map, b, x, BC data,
    solver scratch (6 vectors, an FP32 copy of the values and, for vector P2,
    its block-column index), coefficients."""
    s = problem_sizes(kind, n)
    ncoef = 2 if kind == "vp2" else 1
    return (8 * s["nnz"] + s["cells"] * s["k"] * s["k"] + 8 * 2 * s["rows"] + 9 * s["rows"] + 8 * 6 * s["rows"]
            + 4 * s["nnz"] + (s["nnz"] // 9 * 4 + s["rows"] // 3 * 4 if kind == "vp2" else 0)
            + 8 * ncoef * s["cells"])


def shared_bytes(kind: str, n: int) -> int:
    """Device bytes shared by all slots of one (family, n): CSR pattern,
    dofmaps and mesh."""
    s = problem_sizes(kind, n)
    return 4 * (s["nnz"] + s["rows"] + 1) + 4 * s["rows"] + 4 * s["k"] * s["cells"] + 16 * s["cells"] + \
        24 * s["vertices"] + 16 * s["cells"]


def make_requests(count: int, rate: float, seed: int = 0, nmin: int = 8, nmax: int = 96,
                  mix=(0.35, 0.35, 0.30), rtol: float = 1e-8, materialize: bool = True) -> list:
    """Poisson-process arrivals at `rate` req/s; 35% P1 / 35% P2 Poisson, 30%
    vector-P2 elasticity; n log-uniform in [nmin, nmax]; lognormal DG0
    coefficients (k = exp N(0,1); lam = 0.5 exp N(0,1), mu = 0.2 exp N(0,1)).
    ``materialize=False`` leaves ``coef`` empty (the coefficient arrays of a
    long request stream can exceed host memory)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count) if rate > 0 else np.zeros(count)
    arrivals = np.cumsum(gaps) - gaps[0]
    kinds = rng.choice(FAMILIES, size=count, p=list(mix))
    ns = np.rint(np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=count))).astype(int)
    out = []
    for i in range(count):
        coef = ()
        if materialize:
            C = 6 * int(ns[i]) ** 3
            if kinds[i] == "vp2":
                coef = (0.5 * np.exp(rng.standard_normal(C)), 0.2 * np.exp(rng.standard_normal(C)))
            else:
                coef = (np.exp(rng.standard_normal(C)),)
        out.append(Request(i, str(kinds[i]), int(ns[i]), coef, float(arrivals[i]), rtol))
    return out


def percentile(values, q):
    if not values:
        return None
    return float(np.percentile(np.asarray(values), q))


# ---------------------------------------------------------------------------
# admission (host logic; no device work, tested on CPU)
# ---------------------------------------------------------------------------
class SlotLedger:
    """Device-memory accounting for slots and shared per-size data.

    ``reserve(key, nbytes, shared)`` returns "reuse" (an idle slot of the key),
    "new" (bytes reserved, after evicting idle slots of other keys least
    recently used first), "wait" (not enough memory now) or "never" (more
    than the whole budget)."""

    def __init__(self, budget: int):
        self.budget = int(budget)
        self.idle: "collections.OrderedDict[tuple, list]" = collections.OrderedDict()
        self.slot_size: dict = {}
        self.shared: dict = {}        # key -> bytes of shared data (present while any slot of the key exists)
        self.slots_of: collections.Counter = collections.Counter()
        self.used = 0
        self.peak = 0
        self.evicted: list = []

    def _free_key_if_empty(self, key):
        if self.slots_of[key] == 0 and key in self.shared:
            self.used -= self.shared.pop(key)

    def reserve(self, key, nbytes: int, shared: int):
        pool = self.idle.get(key)
        if pool:
            obj = pool.pop()
            if not pool:
                del self.idle[key]
            return "reuse", obj
        need = nbytes + (0 if key in self.shared else shared)
        if need > self.budget:
            return "never", None
        # evict idle slots (least recently released first) until it fits
        while self.used + need > self.budget and self.idle:
            k, pool = next(iter(self.idle.items()))
            obj = pool.pop(0)
            if not pool:
                del self.idle[k]
            self.used -= self.slot_size[id(obj)]
            del self.slot_size[id(obj)]
            self.slots_of[k] -= 1
            self.evicted.append((k, obj))
            self._free_key_if_empty(k)
            need = nbytes + (0 if key in self.shared else shared)
        if self.used + need > self.budget:
            return "wait", None
        if key not in self.shared:
            self.shared[key] = shared
        self.used += need
        self.peak = max(self.peak, self.used)
        self.slots_of[key] += 1
        return "new", None

    def register(self, key, obj, nbytes: int):
        self.slot_size[id(obj)] = nbytes

    def release(self, key, obj, keep: bool = True):
        if keep:
            self.idle.setdefault(key, []).append(obj)
            self.idle.move_to_end(key)
        else:
            self.used -= self.slot_size.pop(id(obj))
            self.slots_of[key] -= 1
            self._free_key_if_empty(key)

    def cancel_new(self, key, nbytes: int):
        """Undo a "new" reservation whose slot could not be built."""
        self.used -= nbytes
        self.slots_of[key] -= 1
        self._free_key_if_empty(key)

    def take_evicted(self):
        out, self.evicted = self.evicted, []
        return out


# ---------------------------------------------------------------------------
# device execution
# ---------------------------------------------------------------------------
class _Shared:
    """Mesh, spaces and pattern of one (family, n), shared by its slots."""

    def __init__(self, kind: str, n: int):
        from . import fem
        self.mesh = fem.create_unit_cube(n)
        if kind == "p1":
            self.V = fem.functionspace(self.mesh, ("P", 1))
        elif kind == "p2":
            self.V = fem.functionspace(self.mesh, ("P", 2))
        else:
            self.V = fem.functionspace(self.mesh, ("P", 2, (3,)))
        self.bc_dofs = fem.locate_boundary_dofs(self.V)
        g = fem.Function(self.V)
        if kind != "vp2":
            g.x.array[:] = self.V.tabulate_dof_coordinates().sum(axis=1)
        self.g = g
        self.sparsity = None


class _Slot:
    """Forms (with their slot maps), matrix, vectors and BCs for one request
    at a time."""

    def __init__(self, kind: str, sh: _Shared, precision: str, asm):
        import torch

        from . import fem
        from .form import form as cuda_form
        from .la import CUDAMatrix, CUDAVector, Sparsity
        C = sh.mesh.num_cells
        dev = asm._ctx.torch_device
        self.coef = [torch.empty(C, dtype=torch.float64, device=dev) for _ in range(2 if kind == "vp2" else 1)]
        prec = "fp64" if kind == "p1" else precision
        if kind == "vp2":
            a = fem.elasticity(sh.V, self.coef[0], self.coef[1], precision=prec)
            W3 = fem.functionspace(sh.mesh, ("DG", 0, (3,)))
            L = fem.load(sh.V, fem.Function(W3, np.tile([0.0, 0.0, -1.0], C)))
        else:
            a = fem.stiffness(sh.V, self.coef[0], precision=prec)
            L = fem.load(sh.V, 1.0)
        for c in self.coef:
            c.fill_(1.0)
        self.a = cuda_form(a)
        self.L = cuda_form(L)
        if sh.sparsity is None:
            sh.sparsity = Sparsity.build(asm._ctx, self.a._dofmaps[0], self.a._dofmaps[1])
        self.A = CUDAMatrix(asm._ctx, sh.sparsity)
        self.a._bind(sh.sparsity)
        self.b = CUDAVector(asm._ctx, sh.V.num_dofs)
        self.x = CUDAVector(asm._ctx, sh.V.num_dofs)
        self.bcs = asm.pack_bcs([fem.dirichletbc(sh.g, sh.bc_dofs)])
        self.V = sh.V


def _execute(asm, slot: _Slot, req: Request, variant: str = "auto", solver: str = "fp64"):
    import torch
    for dev, host in zip(slot.coef, req.coef):
        dev.copy_(torch.from_numpy(np.ascontiguousarray(host, dtype=np.float64)), non_blocking=True)
    asm.assemble_matrix(slot.a, slot.A, bcs=slot.bcs, variant=variant)
    asm.assemble_rhs(slot.L, slot.a, slot.bcs, vec=slot.b)
    slot.x.vector.zero_()
    if solver == "mixed" and slot.V.bs != 3:
        solver = "fp64"  # scalar systems: the FP64 solve is the faster one
    x, its, res = asm.solve(slot.A, slot.b, slot.x, rtol=req.rtol, raise_on_failure=False, precision=solver,
                            block_size=slot.V.bs)
    xh = x.vector.to("cpu")  # waits for this stream only
    return xh.numpy(), its, res


class Server:
    """Continuous-batching assemble-and-solve server.

    ``workers``: concurrent requests on the device (one stream each).
    ``hbm_budget``: bytes the server may hold for slots and shared data.
    ``precision``: element tensors of the P2 and vector-P2 forms ("fp32" or
    "fp64"; P1 is always FP64).  ``variant``: matrix assembly variant
    ("deterministic" makes every result bitwise independent of what else
    runs).  ``solver``: "mixed" (vector P2: FP32 values in 3x3 blocks in the
    inner PCG iterations, refined in FP64 to the request's rtol; P1 / P2:
    FP64) or "fp64".
    ``plain=True``: the one-at-a-time FP64 path (one worker, nothing cached,
    FP64 solver)."""

    def __init__(self, workers: int = 4, hbm_budget: int = 40 << 30, precision: str = "fp32", plain: bool = False,
                 variant: str = "auto", solver: str = "mixed"):
        import torch

        from .assemble import CUDAAssembler
        self.plain = plain
        self.variant = variant
        self.workers = 1 if plain else int(workers)
        self.precision = "fp64" if plain else precision
        self.solver = "fp64" if plain else solver
        self.ledger = SlotLedger(hbm_budget)
        self._shared: dict = {}
        self._shared_lock = threading.Lock()
        self._key_locks: dict = collections.defaultdict(threading.Lock)
        self._asm = CUDAAssembler()
        self._device = torch.cuda.current_device()
        self._streams = [torch.cuda.Stream() for _ in range(self.workers)]
        self.max_concurrent = 0

    # -- caches ---------------------------------------------------------------
    def _shared_for(self, key):
        with self._key_locks[key]:
            sh = self._shared.get(key)
            if sh is None:
                sh = _Shared(*key)
                if not self.plain:
                    self._shared[key] = sh
            return sh

    def _drop_evicted(self):
        from . import release_caches
        for key, slot in self.ledger.take_evicted():
            del slot
            if self.ledger.slots_of[key] == 0:
                sh = self._shared.pop(key, None)
                if sh is not None:
                    release_caches(sh.mesh)

    def warm(self, keys):
        """Build one slot per (family, n) ahead of traffic, within the budget."""
        import torch
        with torch.cuda.stream(self._streams[0]):
            for key in keys:
                nb, sb = slot_bytes(*key), shared_bytes(*key)
                st, _ = self.ledger.reserve(key, nb, sb)
                if st != "new":
                    continue
                slot = _Slot(key[0], self._shared_for(key), self.precision, self._asm)
                self.ledger.register(key, slot, nb)
                self.ledger.release(key, slot, keep=True)
        torch.cuda.synchronize()

    # -- serving --------------------------------------------------------------
    def run(self, requests: typing.Sequence[Request], realtime: bool = True) -> list:
        """Serve `requests` (arrival times relative to the start; ``realtime``
        waits for them).  Returns the results in request order."""
        import torch

        pending: collections.deque = collections.deque()
        cond = threading.Condition()
        results: dict = {}
        state = {"arrived": 0, "active": 0}
        t0 = time.perf_counter()
        total = len(requests)

        def worker(wid):
            torch.cuda.set_device(self._device)
            stream = self._streams[wid]
            while True:
                with cond:
                    while True:
                        if pending:
                            req = pending[0]
                            nb, sb = slot_bytes(*req.key), shared_bytes(*req.key)
                            if self.plain:
                                status, slot = self.ledger.reserve(("plain",) + req.key, nb, sb)
                            else:
                                status, slot = self.ledger.reserve(req.key, nb, sb)
                            if status == "never":
                                pending.popleft()
                                now = time.perf_counter() - t0
                                results[req.rid] = Result(req.rid, req.kind, req.n, None, 0, float("nan"),
                                                          req.arrival, now, now,
                                                          error="request larger than the device-memory budget")
                                cond.notify_all()
                                continue
                            if status in ("reuse", "new"):
                                pending.popleft()
                                break
                        if state["arrived"] == total and not pending:
                            return
                        cond.wait(0.05)
                    state["active"] += 1
                    self.max_concurrent = max(self.max_concurrent, state["active"])
                    self._drop_evicted()
                admitted = time.perf_counter() - t0
                key = ("plain",) + req.key if self.plain else req.key
                err = None
                try:
                    with torch.cuda.stream(stream):
                        if slot is None:
                            try:
                                slot = _Slot(req.kind, self._shared_for(req.key), self.precision, self._asm)
                            except Exception:
                                with cond:
                                    self.ledger.cancel_new(key, nb)
                                raise
                            with cond:
                                self.ledger.register(key, slot, nb)
                        x, its, res = _execute(self._asm, slot, req, self.variant, self.solver)
                except Exception as e:  # the request fails, the server goes on
                    x, its, res, err = None, 0, float("nan"), f"{type(e).__name__}: {e}"
                done = time.perf_counter() - t0
                with cond:
                    results[req.rid] = Result(req.rid, req.kind, req.n, x, its, res, req.arrival, admitted, done, err)
                    if slot is not None:
                        self.ledger.release(key, slot, keep=not self.plain)
                    state["active"] -= 1
                    cond.notify_all()
                if self.plain:
                    from . import release_caches
                    mesh = slot.V.mesh if slot is not None else None
                    slot = None
                    if mesh is not None:
                        release_caches(mesh)
                    torch.cuda.synchronize()

        threads = [threading.Thread(target=worker, args=(w,), daemon=True) for w in range(self.workers)]
        for th in threads:
            th.start()
        for req in sorted(requests, key=lambda r: r.arrival):
            if realtime:
                delay = req.arrival - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            with cond:
                pending.append(req)
                state["arrived"] += 1
                cond.notify_all()
        for th in threads:
            th.join()
        torch.cuda.synchronize()
        return [results[r.rid] for r in requests]


def summarize(results: typing.Sequence[Result]) -> dict:
    ok = [r for r in results if r.error is None]
    lat = [r.latency for r in ok]
    span = max((r.done for r in results), default=0.0) - min((r.arrival for r in results), default=0.0)
    return {"requests": len(results), "completed": len(ok), "errors": len(results) - len(ok),
            "throughput_rps": len(ok) / span if span > 0 else None,
            "p50_ms": None if not lat else 1e3 * percentile(lat, 50),
            "p99_ms": None if not lat else 1e3 * percentile(lat, 99),
            "mean_iterations": float(np.mean([r.iterations for r in ok])) if ok else None,
            "makespan_s": span}


def solution_difference(a: Result, b: Result) -> float:
    if a.x is None or b.x is None:
        return math.inf
    return float(np.linalg.norm(a.x - b.x) / max(np.linalg.norm(b.x), 1e-300))
