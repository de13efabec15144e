#!/usr/bin/env python
"""Headline benchmark: FEM system assembly on one B200 (matrix nnz/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload p2|p2mid|p1|p1big|vp2|p3|batch|multimesh|serve|blocksys|interp|dg] [--variant auto|tile|atomic|sorted-slot]

Default workload (the configuration the headline metric is quoted on): P2
Poisson on the unit cube, 96^3 hexes x 6 = 5,308,416 tets, 7,189,057 dofs,
nnz 204,763,393, k a P1 field with log k ~ N(0,1) per vertex, f DG0 ~ U[-1,1],
Dirichlet g = x+y+z on the whole boundary with lifting; FP64.

One step = zero A, assemble A with BC rows/cols skipped and unit diagonal,
assemble b, apply lifting, set_bc (the five calls of the reference's
examples/poisson.py timing loop).  ``value`` = nnz per second of whole steps
with all inputs resident in HBM (CUDA events on the launching stream, max over
ranks); ``e2e`` = the same through the public Python API with host buffers:
the coefficient upload (H2D, pinned) that the reference performs on every
assemble call and the read-back of b (D2H) are inside the timed region.
The CSR value array (1.64 GB) exceeds the 126 MB L2, so no flush is needed
between steps.

Multi-GPU: replicas only (the assembly path runs on one GPU with no ghost
exchange); each rank assembles its own copy, value = N * nnz / max step time.
``--impl reference`` times the C restatement of the reference's CPU path
(oracle/cfem.c: per-cell tabulation, binary-search CSR insertion, row-owning
threads) with all host threads on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cuda-dolfinx_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

WORKLOADS = {
    "p2": dict(kind="p2", n=96, precision="fp64",
               desc="P2 Poisson n=96: 5,308,416 tets, k P1 lognormal, f DG0 U[-1,1], g=x+y+z"),
    "p2mid": dict(kind="p2", n=48, precision="fp64",
                  desc="P2 Poisson n=48 (profiling size): 663,552 tets, k P1 lognormal, f DG0, g=x+y+z"),
    "p1": dict(kind="p1", n=32, precision="fp64",
               desc="P1 Poisson n=32: 196,608 tets, k=1, f=P1(sin sin sin), homogeneous Dirichlet"),
    "p1big": dict(kind="p1", n=128, precision="fp64",
                  desc="P1 Poisson n=128: 12,582,912 tets, k=1, f=P1(sin sin sin), homogeneous Dirichlet"),
    "vp2": dict(kind="vp2", n=64, precision="fp32",
                desc="vector-P2 elasticity n=64: 1,572,864 jittered tets, lam/mu DG0, FP32 element tensors"),
    "vp2mid": dict(kind="vp2", n=32, precision="fp32",
                   desc="vector-P2 elasticity n=32 (profiling size): 196,608 jittered tets, lam/mu DG0, FP32 element "
                        "tensors"),
    "p3": dict(kind="p3", n=48, precision="fp64",
               desc="equispaced P3 Poisson n=48: 663,552 tets, 3,048,625 dofs, k DG0 lognormal, f DG0 U[-1,1], "
                    "g=x+y+z"),
    "p3mid": dict(kind="p3", n=32, precision="fp64",
                  desc="equispaced P3 Poisson n=32 (profiling size): 196,608 tets, k DG0 lognormal, f DG0, g=x+y+z"),
}
# batched workload: many DG0-coefficient instances on one mesh and pattern
BATCH = dict(n=48, instances=256, cpu_sample=4,
             desc="256 instances of P1 Poisson on one 48^3 x 6 = 663,552-tet mesh, DG0 k log-uniform "
                  "[1e-2,1e2] per cell and instance, one shared pattern, homogeneous Dirichlet; FP32 element "
                  "tensors, FP64 accumulation")
# kernels of one batched call with <= 384 instances: one cooperative persistent kernel (coefficient
# pack, grid barrier, gather); the unit element tensors and slot records are built once per mesh
BATCH_KERNELS = 1
# many independent meshes in one captured graph
MULTI = dict(count=64, nmin=8, nmax=64, cpu_every=8,
             desc="64 unit-cube tet meshes, n^3 x 6 cells with n ~ U{8..64} (seeded), P1 (k=1) and P2 (k P1 "
                  "lognormal) 50/50, Dirichlet on the boundary; P2 element tensors FP32, P1 FP64, FP64 "
                  "accumulation; all matrix assemblies in one CUDA graph, variant per item from the autotuner")
# serving: assemble-and-solve requests with Poisson arrivals
SERVE = dict(requests=120, rates=(50.0, 200.0, 1000.0), nmin=8, nmax=48, workers=4, budget_gb=60,
             desc="assemble + Jacobi-PCG (rtol 1e-8) requests with Poisson arrivals; 35% P1 / 35% P2 Poisson "
                  "(k DG0 lognormal, f=1, g=x+y+z), 30% vector-P2 elasticity (lam, mu DG0 lognormal, body force "
                  "(0,0,-1), u=0); unit-cube meshes n^3 x 6 tets, n log-uniform")
L2_BYTES = 126 * 1024 * 1024
# kernels of one step besides the matrix call: zero b, the lifting, then the
# element vectors + set_bc in one kernel (fe_assemble_rhs); 4 with the three
# separate calls (--rhs calls)
VECTOR_KERNELS = 3


def matrix_kernels(kind: str, variant: str, big: bool = False, nnz: int = 1 << 30) -> int:
    """Kernel launches of one fe_assemble_matrix call (with BCs): 2 for the
    single-pass variants (row gather, tile, ordered tile: kernel +
    set_diagonal) and for the scatters after the zero pass that also writes
    the BC diagonal (coalesced, block, atomic with both reductions: zero +
    kernel), 3 with the upper-triangle scatter (zero + scatter + transpose
    pass) and for the sorted-slot reduction (element tensors + gather +
    set_diagonal)."""
    if variant in ("tile", "row-gather") or (variant == "deterministic" and kind in ("p1", "p2")):
        return 2
    if variant in ("sorted-slot", "deterministic"):
        return 3
    atomic = variant == "atomic" or (variant == "auto" and not (kind == "p1" and big)
                                     and kind not in ("p2", "vp2", "p3"))
    if kind in ("p1", "vp2", "p3") and atomic:
        return 3  # zero + upper-triangle scatter + lower-triangle transpose
    return 2  # zero (with the BC diagonal) + kernel


_PINNED: list = []


def reduce_over_ranks(values, op: str = "max", device: str = "cuda"):
    """Element-wise max (timings) or min (throughputs) of per-rank values;
    every rank gets the result; the identity without a process group."""
    import torch
    import torch.distributed as dist

    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.MIN)
    return [float(x) for x in t]


def replica_rate(units_per_rank: float, steps: int, max_ms: float, world: int) -> float:
    """Whole-job throughput of N replicas: all ranks' units over the slowest
    rank's time."""
    return world * units_per_rank * steps / (max_ms / 1e3)


# ---------------------------------------------------------------------------
# problem construction (host, seeded)
# ---------------------------------------------------------------------------
def make_inputs(kind: str, n: int, seed: int = 0, pinned: bool = False, precision: str = "fp64"):
    """Seeded synthetic inputs with the shapes of the benchmark configuration
    (``precision`` applies to the P2 stiffness form)."""
    from cudolfinx import fem

    rng = np.random.default_rng(seed)
    mesh = fem.create_unit_cube(n, jitter=0.2 if kind == "vp2" else 0.0, seed=seed)
    C = mesh.num_cells

    def host(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if not pinned:
            return a
        import torch
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        _PINNED.append(t)  # keep the pinned buffer alive with its numpy view
        out = t.numpy()
        out[...] = a
        return out

    I = {"kind": kind, "n": n, "mesh": mesh}
    if kind == "p1":
        V = fem.functionspace(mesh, ("P", 1))
        X = V.tabulate_dof_coordinates()
        f = fem.Function(V)
        f.x.array = host(np.sin(np.pi * X[:, 0]) * np.sin(np.pi * X[:, 1]) * np.sin(np.pi * X[:, 2]))
        a = fem.stiffness(V, 1.0)
        L = fem.load(V, f)
        g = fem.Function(V)
        I.update(k=None, f=f.x.array, g=g.x.array)
    elif kind == "p2":
        V = fem.functionspace(mesh, ("P", 2))
        V1 = fem.functionspace(mesh, ("P", 1))
        W = fem.functionspace(mesh, ("DG", 0))
        k = fem.Function(V1)
        k.x.array = host(np.exp(rng.standard_normal(V1.num_dofs)))
        f = fem.Function(W)
        f.x.array = host(rng.uniform(-1.0, 1.0, size=C))
        g = fem.Function(V)
        g.x.array[:] = V.tabulate_dof_coordinates().sum(axis=1)
        a = fem.stiffness(V, k, precision=precision)
        L = fem.load(V, f)
        I.update(k=k.x.array, f=f.x.array, g=g.x.array)
    elif kind == "p3":
        V = fem.functionspace(mesh, ("P", 3))
        W = fem.functionspace(mesh, ("DG", 0))
        k = fem.Function(W)
        k.x.array = host(np.exp(rng.standard_normal(C)))
        f = fem.Function(W)
        f.x.array = host(rng.uniform(-1.0, 1.0, size=C))
        g = fem.Function(V)
        g.x.array[:] = V.tabulate_dof_coordinates().sum(axis=1)
        a = fem.stiffness(V, k, precision=precision)
        L = fem.load(V, f)
        I.update(k=k.x.array, f=f.x.array, g=g.x.array)
    elif kind == "vp2":
        V = fem.functionspace(mesh, ("P", 2, (3,)))
        W = fem.functionspace(mesh, ("DG", 0))
        W3 = fem.functionspace(mesh, ("DG", 0, (3,)))
        lam = fem.Function(W)
        lam.x.array = host(rng.uniform(0.5, 2.0, size=C))
        mu = fem.Function(W)
        mu.x.array = host(rng.uniform(0.2, 1.0, size=C))
        f = fem.Function(W3)
        f.x.array = host(np.tile([0.0, 0.0, -1.0], C))
        a = fem.elasticity(V, lam, mu, precision="fp32")
        L = fem.load(V, f)
        g = fem.Function(V)
        I.update(lam=lam.x.array, mu=mu.x.array, f=f.x.array, g=g.x.array)
    else:
        raise ValueError(kind)
    bc_dofs = fem.locate_boundary_dofs(V)
    bc = fem.dirichletbc(g, bc_dofs)
    I.update(V=V, a=a, L=L, bc=bc, bc_dofs=bc_dofs, ndof=V.num_nodes, bs=V.bs, dofs=V.dofs,
             coords=mesh.geometry_x, cells=mesh.cells)
    return I


def host_pattern(I):
    """CSR pattern on the host (same builder as the device path; bit-exact with
    the oracle in tests/test_host.py)."""
    from cudolfinx import _lib

    d = np.ascontiguousarray(I["dofs"], dtype=np.int32)
    nnz = ctypes.c_int64()
    rp, cl = ctypes.c_void_p(), ctypes.c_void_p()
    _lib.check(_lib.lib.fe_pattern_build_host(d.ctypes.data, d.ctypes.data, d.shape[0], d.shape[1], d.shape[1],
                                              I["bs"], I["bs"], I["ndof"], I["ndof"], ctypes.byref(nnz),
                                              ctypes.byref(rp), ctypes.byref(cl)), "fe_pattern_build_host")
    nrows = I["ndof"] * I["bs"]
    row_ptr = np.ctypeslib.as_array((ctypes.c_int32 * (nrows + 1)).from_address(rp.value)).copy()
    col = np.ctypeslib.as_array((ctypes.c_int32 * nnz.value).from_address(cl.value)).copy()
    _lib.lib.fe_free_host(rp)
    _lib.lib.fe_free_host(cl)
    return row_ptr, col


def oracle_problem(I):
    P = {"kind": I["kind"], "n": I["n"], "coords": I["coords"], "cells": I["cells"], "dofs": I["dofs"],
         "bs": I["bs"], "ndof": I["ndof"], "bc_dofs": I["bc_dofs"], "g": I["g"], "f": I["f"]}
    if I["kind"] == "vp2":
        P.update(lam=I["lam"], mu=I["mu"], f=np.asarray(I["f"]).reshape(-1, 3))
    else:
        P["k"] = I.get("k")
    return P


# ---------------------------------------------------------------------------
# CPU legs (C restatement of the reference algorithm)
# ---------------------------------------------------------------------------
def workload_config(W, cells, dofs, nnz, world):
    """The `config` object of both arms (identical for the same workload)."""
    return {"workload": W["desc"], "cells": int(cells), "dofs": int(dofs), "nnz": int(nnz),
            "step": "zero A + assemble A (BC skip, unit diagonal) + assemble b + lifting + set_bc",
            "l2": ("inputs larger than L2 (CSR values %.2f GB), no flush between steps" % (8 * nnz / 1e9))
            if 8 * nnz > L2_BYTES else ("working set fits in L2 (CSR values %.1f MB), no flush: steps time "
                                        "L2-resident latency" % (8 * nnz / 1e6)),
            "parallelism": f"replicas x{world}"}


def cpu_assembler(I, row_ptr, col):
    from oracle import cfem

    threads = os.cpu_count() or 1
    return cfem.CpuAssembler(oracle_problem(I), row_ptr, col, nthreads=threads), threads


def cpu_step(C):
    t0 = time.perf_counter()
    C.assemble_matrix()
    C.assemble_rhs()
    return time.perf_counter() - t0


def cpu_baseline(I, row_ptr, col, nnz, reps=2):
    """Times the C restatement on the full workload; returns the baseline
    object and the assembler, which holds the last step's A and b (the
    parity check reads them)."""
    C, threads = cpu_assembler(I, row_ptr, col)
    cpu_step(C)  # warm (page-in, thread start)
    times = [cpu_step(C) for _ in range(reps)]
    t = statistics.median(times)
    return {"value": nnz / t, "unit": "nnz/s", "cores": threads, "kind": "port",
            "sample": f"full workload ({len(I['cells'])} cells, nnz {nnz}): matrix + vector + lifting + set_bc, "
                      f"median of {reps} after 1 warm-up, {threads} threads, C port of the reference CPU "
                      "path (oracle/cfem.c)", "seconds_per_step": t}, C


def parity_report(I, W, A, b, C, row_ptr, col, asm=None, dbc=None):
    """The engine's system at the benchmark size against the C restatement's
    (the cpu_baseline run, same inputs): the CSR pattern against the oracle's
    own builder (bit-exact), A and b entrywise against the per-entry bound
    (1e-12 of the sum of an entry's |contributions| plus 1e-14 of each
    contributing element's largest |entry|; 0 where set_diagonal / set_bc
    write).  FP32 element tensors are reported as the relative Frobenius
    error of A and the Jacobi-PCG solution error against the oracle's FP64
    matrix instead."""
    from oracle import cfem
    from oracle import fem_oracle as fo

    t0 = time.perf_counter()
    rp_o, col_o = cfem.pattern(I["dofs"], I["ndof"], I["bs"])
    pattern_ok = bool(np.array_equal(rp_o, row_ptr) and np.array_equal(col_o, col))
    del rp_o, col_o
    A_gpu = A.values.cpu().numpy()
    b_gpu = b.to_host().copy()
    out = {"oracle": "oracle/cfem.c (C restatement of the reference path), full workload, same inputs",
           "pattern_bit_exact": pattern_ok}
    if W["precision"] == "fp64":
        A_bound = C.matrix_bound()
        okA, wA = fo.within_bound(A_gpu, C.values, A_bound)
        del A_bound
        b_bound = C.rhs_bound()
        okb, wb = fo.within_bound(b_gpu, C.b, b_bound)
        rel = lambda x, y: float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300)) if y.size else 0.0
        out.update({"bound": "per entry: 1e-12 * sum |contributions| + 1e-14 * max|element entry| per "
                             "contributing element; exact where set_diagonal / set_bc write",
                    "A_worst_err_over_bound": wA, "b_worst_err_over_bound": wb,
                    "A_max_abs_err_over_max_abs": rel(A_gpu, C.values), "b_max_abs_err_over_max_abs": rel(b_gpu, C.b),
                    "pass": bool(pattern_ok and okA and okb)})
    else:
        import torch

        import cudolfinx as cx

        ref = torch.from_numpy(C.values).to(A.values.device)
        frob = float(torch.linalg.norm(A.values - ref) / torch.linalg.norm(ref))
        # the oracle's FP64 matrix in the same pattern, both solved on the device
        A64 = cx.CUDAMatrix(asm._ctx, A.sparsity)
        A64.values.copy_(ref)
        del ref
        rtol = 1e-10
        x32, it32, r32 = asm.solve(A, b, rtol=rtol, max_iter=200000, raise_on_failure=False)
        x64, it64, r64 = asm.solve(A64, b, rtol=rtol, max_iter=200000, raise_on_failure=False)
        torch.cuda.synchronize()
        err = float(torch.linalg.norm(x32.vector - x64.vector) / torch.linalg.norm(x64.vector))
        okb, wb = fo.within_bound(b_gpu, C.b, C.rhs_bound())
        out.update({"A_rel_frobenius_vs_oracle_fp64": frob, "solution_rel_error_vs_oracle_fp64": err,
                    "pcg_rtol": rtol, "pcg_iterations": [it32, it64], "b_worst_err_over_bound": wb,
                    "pass": bool(pattern_ok and frob <= 2e-6 and err <= 1e-6 and okb),
                    "bound": "FP32 element tensors: relative Frobenius error <= 2e-6, PCG solution error <= 1e-6 "
                             "(b in FP64 within the per-entry bound)"})
    out["seconds"] = time.perf_counter() - t0
    return out


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# GPU leg
# ---------------------------------------------------------------------------
def algorithmic_matrix_bytes(I, nnz):
    """Bytes one matrix-assembly launch must move (the roofline basis):
    CSR values written once (8/nnz), the cell-to-slot byte map (k^2 per cell),
    the form's cell dofmap (4k per cell), the geometry dofmap (16 per cell),
    coordinates (24 per node), coefficient data, row_ptr (4 per row) and BC
    markers (1 per row)."""
    C = len(I["cells"])
    k = I["dofs"].shape[1]
    nnodes = len(I["coords"])
    nrows = I["ndof"] * I["bs"]
    b = 8 * nnz + k * k * C + 4 * k * C + 16 * C + 24 * nnodes + 4 * (nrows + 1) + nrows
    if I["kind"] == "p2":
        b += 16 * C + 8 * nnodes  # P1 coefficient: its dofmap + vertex values
    elif I["kind"] == "vp2":
        b += 16 * C  # lam, mu DG0
    elif I["kind"] == "p3":
        b += 8 * C  # k DG0
    return b


def load_traffic(kernel_key: str):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh).get(kernel_key)
    except (OSError, ValueError):
        return None


def run_gpu(args, rank, world, local_rank):
    import torch

    import cudolfinx as cx
    from cudolfinx import _lib

    torch.cuda.set_device(local_rank)
    W = WORKLOADS[args.workload]
    t_setup = time.perf_counter()
    I = make_inputs(W["kind"], W["n"], seed=args.seed)
    asm = cx.CUDAAssembler()
    a = cx.form(I["a"])
    L = cx.form(I["L"])
    A = asm.create_matrix(a)
    b = asm.create_vector(L)
    dbc = asm.pack_bcs([I["bc"]])
    hbc = dbc._get_cpp_bcs(I["V"]).handle
    if args.launch:
        cells, stage = (int(v) for v in args.launch.split(","))
        _lib.check(_lib.lib.fe_form_set_launch(a.cuda_form, cells, stage), "fe_form_set_launch")
    nnz = A.sparsity.nnz
    nrows = A.sparsity.num_rows
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    flags = _lib.ASM_ZERO | _lib.VARIANT_FLAGS[args.variant]
    Lib = _lib.lib
    Ap, bp = A.values.data_ptr(), b.vector.data_ptr()

    lift_forms = (ctypes.c_void_p * 1)(a.cuda_form)
    lift_bcs = (ctypes.c_void_p * 1)(hbc)

    def step(ev0=None, ev1=None, st=None, st_vec=None, ev2=None):
        # the matrix call owns its zeroing: a zero pass before the atomic
        # scatter, none for the gather variants (they write every value once);
        # b does not depend on A, so a captured step runs the vector calls on a
        # second stream, concurrently with the matrix
        h = sp if st is None else st
        hv = h if st_vec is None else st_vec
        if ev0 is not None:
            ev0.record(stream)
        _lib.check(Lib.fe_assemble_matrix(a.cuda_form, Ap, hbc, hbc, 1.0, flags, h), "matrix")
        if ev1 is not None:
            ev1.record(stream)
        # b = L - A g on the BC columns, then g on the BC rows
        if args.rhs == "calls":
            _lib.check(Lib.fe_assemble_vector(L.cuda_form, bp, _lib.ASM_ZERO, hv), "vector")
            _lib.check(Lib.fe_apply_lifting(bp, 1, lift_forms, lift_bcs, None, 1.0, hv), "lifting")
            _lib.check(Lib.fe_set_bc(bp, A.sparsity.num_rows, hbc, None, 1.0, hv), "set_bc")
        else:
            _lib.check(Lib.fe_assemble_rhs(L.cuda_form, a.cuda_form, hbc, bp, None, 1.0, _lib.ASM_ZERO, hv), "rhs")
        if ev2 is not None:
            ev2.record(stream)

    step()  # plan build (deterministic), lift-cell list
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    for _ in range(args.warmup):
        step()
    dist = torch.distributed if world > 1 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    mats = [tuple(torch.cuda.Event(enable_timing=True) for _ in range(3)) for _ in range(args.steps)]
    # matrix-call time (roofline basis): eager steps with events around the
    # call; the right-hand side follows it on the same stream
    torch.cuda.nvtx.range_push("timed")  # lets a profiler select these launches (--nvtx-include timed/)
    for k in range(args.steps):
        step(mats[k][0], mats[k][1], ev2=mats[k][2])
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    mat_ms = statistics.mean(m0.elapsed_time(m1) for m0, m1, _ in mats)
    rhs_ms = statistics.mean(m1.elapsed_time(m2) for _, m1, m2 in mats)
    # whole steps: the step's engine calls captured once in a CUDA graph and
    # replayed (every plan and cache exists after the warm-up, so the calls
    # are pure kernel launches); eager steps if the capture is refused
    graph = None
    if not args.no_graph:
        try:
            graph = torch.cuda.CUDAGraph()
            cs = torch.cuda.Stream()
            vs = torch.cuda.Stream()
            cs.wait_stream(stream)
            with torch.cuda.graph(graph, stream=cs):
                vs.wait_stream(cs)  # fork: the vector branch
                step(st=cs.cuda_stream, st_vec=vs.cuda_stream)
                cs.wait_stream(vs)  # join
            stream.wait_stream(cs)
            graph.replay()
            torch.cuda.synchronize()
        except Exception as exc:  # noqa: BLE001 - report and fall back to eager steps
            graph = None
            print(f"graph capture refused ({exc}); timing eager steps", file=sys.stderr)
            torch.cuda.synchronize()
    e_start.record(stream)
    for k in range(args.steps):
        if graph is not None:
            graph.replay()
        else:
            step()
    e_end.record(stream)
    torch.cuda.synchronize()
    total_ms = e_start.elapsed_time(e_end)
    clk = clocks.stop()
    total_ms, mat_ms, rhs_ms = reduce_over_ranks([total_ms, mat_ms, rhs_ms])
    ms_per_step = total_ms / args.steps
    cx.get_cuda_context().synchronize()

    # ---- e2e through the public API with pinned host buffers -------------
    e2e = None
    if not args.no_e2e:
        I2 = make_inputs(W["kind"], W["n"], seed=args.seed, pinned=True)
        a2 = cx.form(I2["a"])
        L2 = cx.form(I2["L"])
        A2 = cx.CUDAMatrix(asm._ctx, A.sparsity)
        b2 = asm.create_vector(L2)
        dbc2 = asm.pack_bcs([I2["bc"]])
        bhost = torch.empty(nrows, dtype=torch.float64, pin_memory=True)
        coef_bytes = sum(np.asarray(c.x.array).nbytes for c in I2["a"].coefficients + I2["L"].coefficients
                         if hasattr(c, "x"))

        vs2 = torch.cuda.Stream()
        # the fork and join cost more than they overlap on launch-bound sizes
        # (P1 n=32: 4.9e9 against 6.4-7.0e9 nnz/s in sequence)
        fork = nnz >= (1 << 22)

        def e2e_step():
            # as in the device leg, the right-hand side (independent of A) on
            # a second stream, concurrent with the matrix; each call uploads
            # its form's host coefficients, b is read back after the RHS
            if not fork:
                asm.assemble_matrix(a2, A2, bcs=dbc2)
                asm.assemble_rhs(L2, a2, dbc2, vec=b2)
                b2.copy_to_host(bhost)
                return
            vs2.wait_stream(stream)
            asm.assemble_matrix(a2, A2, bcs=dbc2)
            with torch.cuda.stream(vs2):
                asm.assemble_rhs(L2, a2, dbc2, vec=b2)
                b2.copy_to_host(bhost)
            stream.wait_stream(vs2)

        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        asm._ctx.join_transfers()  # the last read-back is inside the timed region
        s1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = s0.elapsed_time(s1)
        (e2e_ms,) = reduce_over_ranks([e2e_ms])
        # parity of the two legs (same seeded inputs)
        same = bool(torch.allclose(bhost.to(b.vector.device), b.vector, rtol=1e-12, atol=1e-13))
        e2e = {"value": replica_rate(nnz, args.steps, e2e_ms, world), "unit": "nnz/s",
               "h2d_bytes_per_step": int(coef_bytes), "d2h_bytes_per_step": int(nrows * 8),
               "ms_per_step": e2e_ms / args.steps, "path": "cudolfinx.CUDAAssembler (Python API -> C-ABI)",
               "matches_device_leg": same}

    alg = algorithmic_matrix_bytes(I, nnz)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg / (mat_ms / 1e3) / 1e9
    # the variant "auto" resolves to (fe_assemble_matrix's default): the block
    # kernel for P1 meshes of >= 2^20 cells, the coalesced scatter for P2
    # stiffness, vector-P2 elasticity and FP64 P3 stiffness, the atomic
    # scatter otherwise
    resolved = args.variant
    if resolved == "auto":
        resolved = ("block" if (W["kind"] == "p1" and len(I["cells"]) >= (1 << 20))
                    else "coalesced" if (W["kind"] in ("p2", "vp2") or (W["kind"] == "p3" and W["precision"] == "fp64"))
                    else "atomic")
    kernel_key = f"{args.workload}:{resolved}"
    traffic = load_traffic(kernel_key)
    out = {
        "metric": "matrix nnz/s",
        "value": replica_rate(nnz, args.steps, total_ms, world),
        "unit": "nnz/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if W["precision"] == "fp64" else "f32-element/f64-accumulate",
        "data": "synthetic (seeded numpy inputs with the configuration's shapes and distributions)",
        "config": workload_config(W, len(I["cells"]), nrows, nnz, world),
        "timing": "replays of the step captured in a CUDA graph (matrix and vector branches concurrent)"
        if graph is not None else "eager steps",
        "variant": args.variant,
        "roofline": {"bound": "hbm", "kernel": "matrix assembly (%s%s)" % (args.variant, "" if resolved == args.variant else " = " + resolved),
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "algorithmic_bytes": alg,
                     "kernel_ms": mat_ms, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"
                     if "hbm_gbs" in peaks else "fallback 6650 GB/s"},
        "matrix_nnz_per_s": nnz / (mat_ms / 1e3),
        "rhs_ms": rhs_ms,
        "gpu_launches": (matrix_kernels(W["kind"], args.variant, len(I["cells"]) >= (1 << 20), nnz)
                         + VECTOR_KERNELS + (args.rhs == "calls"))
        * args.steps,
        "clocks": clk,
        "setup_s": setup_s,
    }
    if e2e:
        out["e2e"] = e2e
    if W["precision"] == "fp32" and not args.no_precision:
        out["precision"] = precision_report(I, asm, a, A, b, dbc, args.precision_rtol)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        row_ptr, col = A.sparsity.to_host()
        out["cpu_baseline"], C = cpu_baseline(I, row_ptr, col, nnz)
        if not args.no_parity:
            out["parity"] = parity_report(I, W, A, b, C, row_ptr, col, asm, dbc)
        C.close()
    return out


def precision_report(I, asm, a32, A32, b, dbc, rtol):
    """FP32 element tensors against the FP64 path on the same inputs: relative
    Frobenius error of the matrix, and the relative error of the Jacobi-PCG
    solution (both systems solved to `rtol`)."""
    import torch

    import cudolfinx as cx
    from cudolfinx import fem

    spec = I["a"]
    a64 = cx.form(fem.elasticity(I["V"], *spec.coefficients, precision="fp64") if I["kind"] == "vp2"
                  else fem.stiffness(I["V"], spec.coefficients[0], precision="fp64"))
    A64 = asm.assemble_matrix(a64, cx.CUDAMatrix(asm._ctx, A32.sparsity), bcs=dbc)
    asm.assemble_matrix(a32, A32, bcs=dbc)
    torch.cuda.synchronize()
    frob = float(torch.linalg.norm(A32.values - A64.values) / torch.linalg.norm(A64.values))
    t0 = time.perf_counter()
    x32, it32, r32 = asm.solve(A32, b, rtol=rtol, max_iter=200000, raise_on_failure=False)
    x64, it64, r64 = asm.solve(A64, b, rtol=rtol, max_iter=200000, raise_on_failure=False)
    torch.cuda.synchronize()
    err = float(torch.linalg.norm(x32.vector - x64.vector) / torch.linalg.norm(x64.vector))
    return {"matrix_rel_frobenius_fp32_vs_fp64": frob, "solution_rel_error_fp32_vs_fp64": err,
            "pcg_rtol": rtol, "pcg_iterations": [it32, it64], "pcg_rel_residual": [r32, r64],
            "solve_s": time.perf_counter() - t0,
            "note": "b assembled once (FP64); A with FP32 element tensors (FP64 geometry, exact element row sums) "
                    "vs A with FP64 element tensors; both solved on the device with Jacobi-PCG"}


def batch_inputs(seed: int):
    """P1 stiffness form with a DG0 coefficient on the batch mesh, the BC and
    the oracle-style problem dict (host, seeded)."""
    from cudolfinx import fem

    mesh = fem.create_unit_cube(BATCH["n"])
    V = fem.functionspace(mesh, ("P", 1))
    W = fem.functionspace(mesh, ("DG", 0))
    C = mesh.num_cells
    a = fem.stiffness(V, fem.Function(W, np.ones(C)))
    bc_dofs = fem.locate_boundary_dofs(V)
    bc = fem.dirichletbc(fem.Function(V), bc_dofs)
    I = {"kind": "p1", "n": BATCH["n"], "mesh": mesh, "V": V, "a": a, "bc": bc, "bc_dofs": bc_dofs,
         "ndof": V.num_nodes, "bs": 1, "dofs": V.dofs, "coords": mesh.geometry_x, "cells": mesh.cells,
         "g": np.zeros(V.num_nodes), "f": np.ones(V.num_nodes)}
    return I


def batch_coefficients(S: int, C: int, seed: int, device):
    """k_s(c) log-uniform in [1e-2, 1e2], seeded, generated on the device."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    u = torch.rand((S, C), generator=g, dtype=torch.float64, device=device)
    return torch.exp(np.log(1e-2) + u * (np.log(1e2) - np.log(1e-2)))


def cpu_batch_baseline(I, row_ptr, col, nnz, kd, sample, reps=1):
    """C port of the reference CPU path, one instance at a time (the reference
    has no batch path), on `sample` instances."""
    from oracle import cfem

    threads = os.cpu_count() or 1
    P = oracle_problem(I)
    P["kind"] = "p1k"
    times = []
    for s in range(sample):
        P["k"] = kd[s].cpu().numpy()
        C = cfem.CpuAssembler(P, row_ptr, col, nthreads=threads)
        C.assemble_matrix()  # warm
        t0 = time.perf_counter()
        for _ in range(reps):
            C.assemble_matrix()
        times.append((time.perf_counter() - t0) / reps)
        C.close()
    t = sum(times)
    return {"value": nnz * sample / t, "unit": "nnz/s", "cores": threads, "kind": "port",
            "sample": f"{sample} of the {BATCH['instances']} instances, one matrix assembly each (BC skip, "
                      f"unit diagonal), {threads} threads, C port of the reference CPU path (oracle/cfem.c)",
            "seconds_per_instance": t / sample}


def run_gpu_batch(args, rank, world, local_rank):
    import torch

    import cudolfinx as cx
    from cudolfinx import _lib

    torch.cuda.set_device(local_rank)
    t_setup = time.perf_counter()
    I = batch_inputs(args.seed)
    S = args.instances or BATCH["instances"]
    C = len(I["cells"])
    asm = cx.CUDAAssembler()
    a = cx.form(I["a"])
    A0 = asm.create_matrix(a)
    nnz = A0.sparsity.nnz
    nrows = A0.sparsity.num_rows
    dbc = asm.pack_bcs([I["bc"]])
    hbc = dbc._get_cpp_bcs(I["V"]).handle
    kd = batch_coefficients(S, C, args.seed + 1000 * (rank + 1), "cuda")
    vals = torch.zeros((S, nnz), dtype=torch.float64, device="cuda")
    ktab = (ctypes.c_void_p * S)(*[kd[s].data_ptr() for s in range(S)])
    vtab = (ctypes.c_void_p * S)(*[vals[s].data_ptr() for s in range(S)])
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    Lib = _lib.lib

    def step():
        _lib.check(Lib.fe_assemble_matrix_batch(a.cuda_form, S, ktab, vtab, hbc, hbc, 1.0, _lib.ASM_ZERO, sp),
                   "batch")

    step()
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    for _ in range(args.warmup):
        step()
    dist = torch.distributed if world > 1 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")
    e_start.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    e_end.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    total_ms = e_start.elapsed_time(e_end)
    call_ms = statistics.mean(x.elapsed_time(y) for x, y in ev)
    clk = clocks.stop()

    # the plain path: one FP64 fe_assemble_matrix per instance (default variant)
    ap = cx.form(I["a"])
    ap._bind(A0.sparsity)
    plain_vals = torch.zeros(nnz, dtype=torch.float64, device="cuda")

    def plain_all():
        for s in range(S):
            _lib.check(Lib.fe_form_set_coefficient(ap.cuda_form, 0, _lib.COEFF_DG0, None, kd[s].data_ptr(), C, 1,
                                                   sp), "set_coefficient")
            _lib.check(Lib.fe_assemble_matrix(ap.cuda_form, plain_vals.data_ptr(), hbc, hbc, 1.0, _lib.ASM_ZERO,
                                              sp), "matrix")

    plain_all()
    torch.cuda.synchronize()
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    plain_all()
    p1.record(stream)
    torch.cuda.synchronize()
    plain_ms = p0.elapsed_time(p1)
    # agreement of the last instance between the two paths (FP32 element tensors)
    rel = float(torch.linalg.norm(vals[S - 1] - plain_vals) / torch.linalg.norm(plain_vals))
    total_ms, call_ms, plain_ms = reduce_over_ranks([total_ms, call_ms, plain_ms])

    alg = S * (8 * nnz + 8 * C) + 16 * C + 16 * C + 16 * C + 24 * len(I["coords"]) + 4 * (nrows + 1) + nrows
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg / (call_ms / 1e3) / 1e9
    out = {
        "metric": "matrix nnz/s (batched instances)",
        "value": replica_rate(S * nnz, args.steps, total_ms, world),
        "unit": "nnz/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32-element/f64-accumulate",
        "data": "synthetic (seeded mesh; coefficients from a seeded device generator)",
        "config": {"workload": BATCH["desc"] if S == BATCH["instances"] else
                   BATCH["desc"].replace("256 instances", f"{S} instances"), "instances": S, "cells": C, "dofs": nrows, "nnz": nnz,
                   "step": "fe_assemble_matrix_batch: one persistent launch (pack coefficients, grid barrier, "
                           "gather) into %d CSR value arrays; unit element tensors and slot records built once "
                           "per mesh, before the timed steps" % S,
                   "l2": "inputs larger than L2 (values %.2f GB per step)" % (8 * S * nnz / 1e9),
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "kernel": "batched assembly call (one persistent launch)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": load_traffic("batch"),
                     "algorithmic_bytes": alg, "kernel_ms": call_ms,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                     else "fallback 6650 GB/s"},
        "plain_fp64": {"ms_per_batch": plain_ms, "nnz_per_s": S * nnz / (plain_ms / 1e3),
                       "speedup_of_batch": plain_ms / call_ms,
                       "path": "one fe_assemble_matrix (FP64, default variant) per instance",
                       "rel_frobenius_last_instance": rel},
        "gpu_launches": BATCH_KERNELS * args.steps,
        "clocks": clk,
        "setup_s": setup_s,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        row_ptr, col = A0.sparsity.to_host()
        out["cpu_baseline"] = cpu_batch_baseline(I, row_ptr, col, nnz, kd, BATCH["cpu_sample"])
    return out


# two-field block system with a restricted second field
BLOCKSYS = dict(n=64, cpu_n=16,
                desc="two-field P2 block system on the unit cube, n=64 (1,572,864 tets): [[K, -K], [-K, 2K]] with "
                     "K = k grad.grad, k P1 lognormal, the second field restricted to the dofs with x <= 1/2, "
                     "Dirichlet g=x+y+z (2g) on the boundary of both fields, loads f DG0 U[-1,1]; FP64")
# launches of one block step: zero A + 4 x (scatter + set_diagonal) + zero b + 2 loads
BLOCKSYS_KERNELS = 12


def blocksys_inputs(n: int, seed: int, pinned: bool = False):
    """Forms, BCs and oracle-side arrays of the two-field block system."""
    from cudolfinx import fem

    rng = np.random.default_rng(seed)
    mesh = fem.create_unit_cube(n)
    C = mesh.num_cells
    V = fem.functionspace(mesh, ("P", 2))
    W = fem.functionspace(mesh, ("P", 2))
    V1 = fem.functionspace(mesh, ("P", 1))
    DG = fem.functionspace(mesh, ("DG", 0))

    def host(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if not pinned:
            return a
        import torch
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        _PINNED.append(t)
        out = t.numpy()
        out[...] = a
        return out

    k = np.exp(rng.standard_normal(V1.num_dofs))
    f = rng.uniform(-1.0, 1.0, size=C)
    X = V.tabulate_dof_coordinates()
    R = np.nonzero(X[:, 0] <= 0.5 + 1e-12)[0].astype(np.int32)
    kf = [fem.Function(V1, host(k)), fem.Function(V1, host(-k)), fem.Function(V1, host(-k)),
          fem.Function(V1, host(2 * k))]
    a = [[fem.stiffness(V, kf[0]), fem.stiffness(V, kf[1], trial=W)],
         [fem.stiffness(W, kf[2], trial=V), fem.stiffness(W, kf[3])]]
    L = [fem.load(V, fem.Function(DG, host(f))), fem.load(W, fem.Function(DG, host(f)))]
    g = X.sum(axis=1)
    bnd = fem.locate_boundary_dofs(V)
    bcs = [fem.dirichletbc(fem.Function(V, g), bnd), fem.dirichletbc(fem.Function(W, 2 * g), bnd)]
    return dict(mesh=mesh, V=V, W=W, a=a, L=L, bcs=bcs, R=R, k=k, f=f, bnd=bnd, cells=mesh.cells,
                coords=mesh.geometry_x, dofs=V.dofs, ndof=V.num_nodes)


def blocksys_alg_bytes(I, nnz, rows):
    """Algorithmic bytes of the block matrix assembly: values written once
    (8/nnz) and, per block, its byte map (100/cell), test and trial dofmaps
    (80/cell), geometry dofmap (16/cell), coordinates (24/node), the P1
    coefficient (16/cell + 8/node), segment starts (4/row) and BC markers
    (1/row + 1/column)."""
    C, nv = len(I["cells"]), len(I["coords"])
    nV, nW = I["ndof"], len(I["R"])
    b = 8 * nnz
    for r, c in ((nV, nV), (nV, nW), (nW, nV), (nW, nW)):
        b += 100 * C + 80 * C + 16 * C + 24 * nv + 16 * C + 8 * nv + 4 * (r + 1) + r + c
    return b


def blocksys_cpu_sample(n: int, seed: int, steps: int = 1):
    """Oracle (numpy) restatement of the block system on the n-sized mesh:
    element tensors + block matrix + block vector per step; returns
    (seconds per step, monolithic nnz)."""
    from oracle import fem_oracle as fo

    coords, cells = fo.unit_cube_tet_mesh(n)
    dofs, nd, grid = fo.p2_dofmap(n, cells)
    rng = np.random.default_rng(seed)
    k = np.exp(rng.standard_normal((n + 1) ** 3))
    f = rng.uniform(-1.0, 1.0, size=len(cells))
    X = fo.dof_coordinates(coords, cells, dofs, nd, 2)
    R = np.nonzero(X[:, 0] <= 0.5 + 1e-12)[0]
    bnd = fo.boundary_dofs_from_grid(grid, 2 * n)
    mk = np.zeros(nd, dtype=np.uint8)
    mk[bnd] = 1
    dr = fo.restricted_dofmap(dofs, R, nd)
    mkr = mk[R]
    bcr = np.nonzero(mkr)[0]
    parts = [(dofs, dofs, 1, 1, 0, 0), (dofs, dr, 1, 1, 0, nd), (dr, dofs, 1, 1, nd, 0), (dr, dr, 1, 1, nd, nd)]
    rp, col = fo.block_pattern(parts, nd + len(R), nd + len(R))
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        K = fo.p2_stiffness(coords, cells, k[cells])
        B = [dict(Ae=K, dofs0=dofs, dofs1=dofs, row_offset=0, col_offset=0, markers0=mk, markers1=mk, bc_rows=bnd),
             dict(Ae=-K, dofs0=dofs, dofs1=dr, row_offset=0, col_offset=nd, markers0=mk, markers1=mkr, bc_rows=bnd),
             dict(Ae=-K, dofs0=dr, dofs1=dofs, row_offset=nd, col_offset=0, markers0=mkr, markers1=mk, bc_rows=bcr),
             dict(Ae=2 * K, dofs0=dr, dofs1=dr, row_offset=nd, col_offset=nd, markers0=mkr, markers1=mkr,
                  bc_rows=bcr)]
        for b in B:
            b.update(bs0=1, bs1=1)
        fo.assemble_block_matrix(B, rp, col)
        be = fo.p2_load_dg0(coords, cells, f)
        fo.assemble_block_vector([(be, dofs, 1, 0), (be, dr, 1, nd)], nd + len(R))
        times.append(time.perf_counter() - t0)
    return statistics.median(times), len(col)


def run_gpu_blocksys(args, rank, world, local_rank):
    import torch

    import cudolfinx as cx
    from cudolfinx import _lib

    torch.cuda.set_device(local_rank)
    t_setup = time.perf_counter()
    I = blocksys_inputs(BLOCKSYS["n"], args.seed)
    asm = cx.CUDAAssembler()
    A = cx.form(I["a"], restriction=([None, I["R"]], [None, I["R"]]))
    Lb = cx.form(I["L"], restriction=[None, I["R"]])
    M = asm.create_matrix_block(A)
    b = asm.create_vector_block(Lb)
    dbc = asm.pack_bcs(I["bcs"])
    nnz, nrows = M.sparsity.nnz, M.sparsity.num_rows
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    Lib = _lib.lib
    blocks = []
    for i, row in enumerate(A.forms):
        for j, f in enumerate(row):
            h0 = dbc._get_cpp_bcs(f.function_spaces[0], f.restriction(0))
            h1 = dbc._get_cpp_bcs(f.function_spaces[1], f.restriction(1))
            blocks.append((f.cuda_form, h0.handle if h0 else None, h1.handle if h1 else None))
    vforms = [(f.cuda_form, off) for f, off in zip(Lb.forms, Lb.offsets)]
    Mp, bp = M.values.data_ptr(), b.vector.data_ptr()

    def step(ev0=None, ev1=None):
        if ev0 is not None:
            ev0.record(stream)
        _lib.check(Lib.fe_zero_entries(Mp, nnz, sp), "zero")
        for h, b0, b1 in blocks:
            _lib.check(Lib.fe_assemble_matrix(h, Mp, b0, b1, 1.0, 0, sp), "matrix block")
        if ev1 is not None:
            ev1.record(stream)
        _lib.check(Lib.fe_zero_entries(bp, nrows, sp), "zero b")
        for h, off in vforms:
            _lib.check(Lib.fe_assemble_vector(h, bp + 8 * off, 0, sp), "vector block")

    step()
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    for _ in range(args.warmup):
        step()
    dist = torch.distributed if world > 1 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    mats = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        step(*mats[k])
    e1.record(stream)
    torch.cuda.synchronize()
    total_ms = e0.elapsed_time(e1)
    mat_ms = statistics.mean(x.elapsed_time(y) for x, y in mats)
    clk = clocks.stop()
    total_ms, mat_ms = reduce_over_ranks([total_ms, mat_ms])

    e2e = None
    if not args.no_e2e:
        I2 = blocksys_inputs(BLOCKSYS["n"], args.seed, pinned=True)
        A2 = cx.form(I2["a"], restriction=([None, I2["R"]], [None, I2["R"]]))
        L2 = cx.form(I2["L"], restriction=[None, I2["R"]])
        M2 = cx.CUDAMatrix(asm._ctx, M.sparsity)
        b2 = asm.create_vector_block(L2)
        dbc2 = asm.pack_bcs(I2["bcs"])
        bhost = torch.empty(nrows, dtype=torch.float64, pin_memory=True)
        coef_bytes = sum(np.asarray(c.x.array).nbytes for row in I2["a"] for f in row for c in f.coefficients) + \
            sum(np.asarray(c.x.array).nbytes for f in I2["L"] for c in f.coefficients)

        def e2e_step():
            asm.assemble_matrix_block(A2, M2, bcs=dbc2)
            asm.assemble_vector_block(L2, b2)
            b2.copy_to_host(bhost)

        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        asm._ctx.join_transfers()  # the last read-back is inside the timed region
        s1.record(stream)
        torch.cuda.synchronize()
        (e2e_ms,) = reduce_over_ranks([s0.elapsed_time(s1)])
        same = bool(torch.allclose(M2.values, M.values, rtol=1e-12, atol=1e-13 * float(M.values.abs().max())))
        e2e = {"value": replica_rate(nnz, args.steps, e2e_ms, world), "unit": "nnz/s",
               "h2d_bytes_per_step": int(coef_bytes), "d2h_bytes_per_step": int(nrows * 8),
               "ms_per_step": e2e_ms / args.steps,
               "path": "cudolfinx.CUDAAssembler.assemble_matrix_block + assemble_vector_block (Python API -> C-ABI)",
               "matches_device_leg": same}

    alg = blocksys_alg_bytes(I, nnz, nrows)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg / (mat_ms / 1e3) / 1e9
    out = {
        "metric": "matrix nnz/s (block system)", "value": replica_rate(nnz, args.steps, total_ms, world),
        "unit": "nnz/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded numpy inputs)",
        "config": {"workload": BLOCKSYS["desc"], "cells": len(I["cells"]), "dofs": nrows, "nnz": nnz,
                   "kept_dofs_second_field": int(len(I["R"])),
                   "step": "zero A + 4 block scatters (BC skip, unit diagonal) + zero b + 2 block loads",
                   "l2": "inputs larger than L2 (values %.2f GB)" % (8 * nnz / 1e9),
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "kernel": "block matrix assembly (zero + 4 blocks)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": load_traffic("blocksys"),
                     "algorithmic_bytes": alg, "kernel_ms": mat_ms,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                     else "fallback 6650 GB/s"},
        "matrix_nnz_per_s": nnz / (mat_ms / 1e3),
        "gpu_launches": BLOCKSYS_KERNELS * args.steps,
        "clocks": clk,
        "setup_s": setup_s,
    }
    if e2e:
        out["e2e"] = e2e
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t, nnz_s = blocksys_cpu_sample(BLOCKSYS["cpu_n"], args.seed, steps=2)
        out["cpu_baseline"] = {"value": nnz_s / t, "unit": "nnz/s", "cores": 1, "kind": "port",
                               "sample": f"the same block system at n={BLOCKSYS['cpu_n']} "
                                         f"({6 * BLOCKSYS['cpu_n'] ** 3} cells, nnz {nnz_s}): element tensors + "
                                         "block matrix + block vector with the numpy oracle (oracle/fem_oracle.py), "
                                         "median of 2, one thread", "seconds_per_step": t}
    return out


def run_reference_blocksys(args):
    steps = max(1, args.steps)
    for _ in range(args.warmup):
        blocksys_cpu_sample(BLOCKSYS["cpu_n"], args.seed, 1)
    t, nnz = blocksys_cpu_sample(BLOCKSYS["cpu_n"], args.seed, steps)
    v = nnz / t
    return {"impl": "reference", "metric": "matrix nnz/s (block system)", "value": v, "unit": "nnz/s",
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": BLOCKSYS["desc"], "sample_n": BLOCKSYS["cpu_n"], "nnz": nnz},
            "cpu_baseline": {"value": v, "unit": "nnz/s", "cores": 1, "kind": "port",
                             "sample": f"n={BLOCKSYS['cpu_n']} block system per step, numpy oracle "
                                       "(the reference's block path needs DOLFINx + PETSc)"},
            "e2e": {"value": v, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# device interpolation: a P2 field into P3 on one mesh
INTERP = dict(n=64, cpu_n=24,
              desc="same-map interpolation P2 -> P3 on the unit cube, n=64 (1,572,864 tets; 2,146,689 source "
                   "and 7,189,057 target dofs), source values N(0,1); FP64")


def run_gpu_interp(args, rank, world, local_rank):
    import torch

    import cudolfinx as cx
    from cudolfinx import _lib, fem

    torch.cuda.set_device(local_rank)
    n = INTERP["n"]
    mesh = fem.create_unit_cube(n)
    V0 = fem.functionspace(mesh, ("P", 2))
    V1 = fem.functionspace(mesh, ("P", 3))
    rng = np.random.default_rng(args.seed)
    c0 = cx.Coefficient(fem.Function(V0, rng.standard_normal(V0.num_dofs)))
    c1 = cx.Coefficient(fem.Function(V1))
    im = fem.interpolation_matrix(V1, V0)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    h1, h0 = c1._dofmap.handle, c0._dofmap.handle
    p1, p0 = c1.device_values.data_ptr(), c0.device_values.data_ptr()

    def step():
        _lib.check(_lib.lib.fe_interpolate(h1, p1, h0, p0, im.ctypes.data, sp), "interpolate")

    step()
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    (ms,) = reduce_over_ranks([e0.elapsed_time(e1)])
    ms_step = ms / args.steps
    n1, n0, C = V1.num_dofs, V0.num_dofs, mesh.num_cells
    # per target dof: owner entry (4) + value written (8); the source values
    # (8 per source dof) and the source dofmap (4 * 10 per cell) read once
    alg = 12 * n1 + 8 * n0 + 40 * C
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg / (ms_step / 1e3) / 1e9
    e2e = None
    if not args.no_e2e:
        host_u0 = torch.from_numpy(c0.values()).pin_memory()
        host_u1 = torch.empty(n1, dtype=torch.float64, pin_memory=True)

        def e2e_step():
            c0.device_values.copy_(host_u0, non_blocking=True)
            step()
            host_u1.copy_(c1.device_values, non_blocking=True)

        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        s1.record(stream)
        torch.cuda.synchronize()
        (e2e_ms,) = reduce_over_ranks([s0.elapsed_time(s1)])
        e2e = {"value": replica_rate(n1, args.steps, e2e_ms, world), "unit": "target dofs/s",
               "h2d_bytes_per_step": 8 * n0, "d2h_bytes_per_step": 8 * n1, "ms_per_step": e2e_ms / args.steps,
               "path": "fe_interpolate with the source uploaded from pinned host memory and the result read back"}
    out = {"metric": "interpolated target dofs/s", "value": replica_rate(n1, args.steps, ms, world),
           "unit": "target dofs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded)",
           "config": {"workload": INTERP["desc"], "cells": C, "source_dofs": n0, "target_dofs": n1,
                      "l2": "working set %.2f GB (> L2)" % (alg / 1e9), "parallelism": f"replicas x{world}"},
           "roofline": {"bound": "hbm", "kernel": "k_interpolate", "achieved": achieved, "peak": peak,
                        "unit": "GB/s", "frac": achieved / peak, "traffic": load_traffic("interp"),
                        "algorithmic_bytes": alg, "kernel_ms": ms_step,
                        "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                        else "fallback 6650 GB/s"},
           "gpu_launches": args.steps, "clocks": clk}
    if e2e:
        out["e2e"] = e2e
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = interp_cpu_sample(INTERP["cpu_n"], args.seed)
    return out


def interp_cpu_sample(n: int, seed: int):
    """The oracle's restatement of the reference algorithm (gather, multiply,
    scatter cell by cell) on the n-sized mesh."""
    from oracle import fem_oracle as fo

    coords, cells = fo.unit_cube_tet_mesh(n)
    d2, n2, _ = fo.p2_dofmap(n, cells)
    d3, n3, _ = fo.p3_dofmap(n, cells)
    u0 = np.random.default_rng(seed).standard_normal(n2)
    im = fo.interpolation_operator(3, 2)
    t0 = time.perf_counter()
    fo.interpolate_same_map(u0, d2, d3, im, n3)
    t = time.perf_counter() - t0
    return {"value": n3 / t, "unit": "target dofs/s", "cores": 1, "kind": "port",
            "sample": f"P2 -> P3 at n={n} ({6 * n ** 3} cells, {n3} target dofs): oracle interpolate_same_map "
                      "(numpy, cell loop in the reference's order), one thread", "seconds_per_step": t}


def run_reference_interp(args):
    r = interp_cpu_sample(INTERP["cpu_n"], args.seed)
    v = r["value"]
    return {"impl": "reference", "metric": "interpolated target dofs/s", "value": v, "unit": "target dofs/s",
            "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * r["seconds_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": INTERP["desc"], "sample_n": INTERP["cpu_n"]},
            "cpu_baseline": r, "e2e": {"value": v, "unit": "target dofs/s", "h2d_bytes_per_step": 0,
                                       "d2h_bytes_per_step": 0}}


# interior-penalty DG1 system: broken P1 stiffness + jump penalty + facet load
DGSYS = dict(n=64, alpha=10.0, cpu_n=16,
             desc="DG1 interior-penalty system on the unit cube, n=64 (1,572,864 tets, 6,291,456 dofs, 3,121,152 "
                  "interior facets): broken P1 stiffness + 10*jump(u)*jump(v)*dS on one union pattern, load "
                  "g*avg(v)*dS with g DG0 U[-1,1]; FP64")
# zero + cell scatter + mirror + jump scatter + vector zero + facet load
DGSYS_KERNELS = 6


def dg_inputs(n: int, seed: int, pinned: bool = False):
    from cudolfinx import fem

    mesh = fem.create_unit_cube(n)
    V = fem.functionspace(mesh, ("DG", 1))
    W = fem.functionspace(mesh, ("DG", 0))
    g = np.random.default_rng(seed).uniform(-1.0, 1.0, mesh.num_cells)
    if pinned:
        import torch
        t = torch.empty(g.shape, dtype=torch.float64, pin_memory=True)
        _PINNED.append(t)
        t.numpy()[:] = g
        g = t.numpy()
    q = fem.interior_facets(mesh)
    a_cell = fem.FormSpec("P1_STIFFNESS", V, [1.0], 2)
    a_jump = fem.jump_penalty(V, DGSYS["alpha"], facets=q)
    L = fem.facet_average_load(V, fem.Function(W, g), facets=q)
    return dict(mesh=mesh, V=V, a_cell=a_cell, a_jump=a_jump, L=L, facets=q, g=g)


def dg_cpu_sample(n: int, seed: int):
    """The oracle on the n-sized DG1 system: element tensors (cells and
    facets) + monolithic matrix + facet load."""
    from oracle import fem_oracle as fo

    coords, cells = fo.unit_cube_tet_mesh(n)
    q = fo.interior_facets(cells)
    C = len(cells)
    d = fo.dg_dofmap(C, 1)
    m = fo.macro_dofmap(d, q)
    N = 4 * C
    g = np.random.default_rng(seed).uniform(-1.0, 1.0, C)
    rp, col = fo.block_pattern([(d, d, 1, 1, 0, 0), (m, m, 1, 1, 0, 0)], N, N)
    t0 = time.perf_counter()
    fo.assemble_block_matrix([
        dict(Ae=fo.p1_stiffness(coords, cells), dofs0=d, dofs1=d, bs0=1, bs1=1, row_offset=0, col_offset=0),
        dict(Ae=fo.interior_jump_tensors(coords, cells, q, 1, np.full(len(q), DGSYS["alpha"])), dofs0=m, dofs1=m,
             bs0=1, bs1=1, row_offset=0, col_offset=0)], rp, col)
    fo.assemble_vector(fo.interior_avg_load(coords, cells, q, 1, fo.facet_average(g, q)), m, N)
    t = time.perf_counter() - t0
    return t, len(col)


def run_gpu_dg(args, rank, world, local_rank):
    import torch

    import cudolfinx as cx
    from cudolfinx import _lib

    torch.cuda.set_device(local_rank)
    t_setup = time.perf_counter()
    I = dg_inputs(DGSYS["n"], args.seed)
    asm = cx.CUDAAssembler()
    a_cell, a_jump, L = cx.form(I["a_cell"]), cx.form(I["a_jump"]), cx.form(I["L"])
    A = asm.create_matrix([a_cell, a_jump])
    b = asm.create_vector(L)
    nnz, nrows = A.sparsity.nnz, A.sparsity.num_rows
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    Lib = _lib.lib
    Ap, bp = A.values.data_ptr(), b.vector.data_ptr()

    def step(ev0=None, ev1=None):
        if ev0 is not None:
            ev0.record(stream)
        _lib.check(Lib.fe_assemble_matrix(a_cell.cuda_form, Ap, None, None, 1.0, _lib.ASM_ZERO, sp), "cell")
        _lib.check(Lib.fe_assemble_matrix(a_jump.cuda_form, Ap, None, None, 1.0, 0, sp), "jump")
        if ev1 is not None:
            ev1.record(stream)
        _lib.check(Lib.fe_assemble_vector(L.cuda_form, bp, _lib.ASM_ZERO, sp), "load")

    step()
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    for _ in range(args.warmup):
        step()
    dist = torch.distributed if world > 1 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    mats = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        step(*mats[k])
    e1.record(stream)
    torch.cuda.synchronize()
    total_ms = e0.elapsed_time(e1)
    mat_ms = statistics.mean(x.elapsed_time(y) for x, y in mats)
    clk = clocks.stop()
    total_ms, mat_ms = reduce_over_ranks([total_ms, mat_ms])

    e2e = None
    if not args.no_e2e:
        I2 = dg_inputs(DGSYS["n"], args.seed, pinned=True)
        c2, j2, L2 = cx.form(I2["a_cell"]), cx.form(I2["a_jump"]), cx.form(I2["L"])
        for f in (c2, j2):
            f._bind(A.sparsity)
        A2 = cx.CUDAMatrix(asm._ctx, A.sparsity)
        b2 = asm.create_vector(L2)
        bhost = torch.empty(nrows, dtype=torch.float64, pin_memory=True)

        def e2e_step():
            asm.assemble_matrix(c2, A2)
            asm.assemble_matrix(j2, A2, zero=False)
            asm.assemble_vector(L2, b2)
            b2.copy_to_host(bhost)

        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        asm._ctx.join_transfers()  # the last read-back is inside the timed region
        s1.record(stream)
        torch.cuda.synchronize()
        (e2e_ms,) = reduce_over_ranks([s0.elapsed_time(s1)])
        same = bool(torch.allclose(A2.values, A.values, rtol=1e-12, atol=1e-13 * float(A.values.abs().max())))
        e2e = {"value": replica_rate(nnz, args.steps, e2e_ms, world), "unit": "nnz/s",
               "h2d_bytes_per_step": int(I2["g"].nbytes), "d2h_bytes_per_step": int(nrows * 8),
               "ms_per_step": e2e_ms / args.steps,
               "path": "cudolfinx.CUDAAssembler.assemble_matrix x2 + assemble_vector (Python API -> C-ABI)",
               "matches_device_leg": same}

    C, nv, F = I["mesh"].num_cells, I["mesh"].num_vertices, len(I["facets"])
    # values once (8/nnz); cell term: byte map 16 + dofmap 16 + geometry 16 per
    # cell, coordinates 24 per vertex; jump term per facet: quad 16, macro dofs
    # 32, byte map 64, both cells' geometry 32; row_ptr 4 per row per launch
    alg = 8 * nnz + 48 * C + 24 * nv + 144 * F + 8 * (nrows + 1)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg / (mat_ms / 1e3) / 1e9
    out = {
        "metric": "matrix nnz/s (DG1 interior penalty)", "value": replica_rate(nnz, args.steps, total_ms, world),
        "unit": "nnz/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": DGSYS["desc"], "cells": C, "dofs": nrows, "nnz": nnz, "interior_facets": F,
                   "step": "cell term (zero + upper-triangle scatter + mirror) + jump term + facet load",
                   "l2": "inputs larger than L2 (values %.2f GB)" % (8 * nnz / 1e9),
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "kernel": "cell + jump matrix assembly", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": load_traffic("dg"),
                     "algorithmic_bytes": alg, "kernel_ms": mat_ms,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                     else "fallback 6650 GB/s"},
        "matrix_nnz_per_s": nnz / (mat_ms / 1e3),
        "gpu_launches": DGSYS_KERNELS * args.steps,
        "clocks": clk,
        "setup_s": setup_s,
    }
    if e2e:
        out["e2e"] = e2e
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t, nnz_s = dg_cpu_sample(DGSYS["cpu_n"], args.seed)
        out["cpu_baseline"] = {"value": nnz_s / t, "unit": "nnz/s", "cores": 1, "kind": "port",
                               "sample": f"the same DG1 system at n={DGSYS['cpu_n']} ({6 * DGSYS['cpu_n'] ** 3} "
                                         f"cells, nnz {nnz_s}): element tensors + matrix + facet load with the numpy "
                                         "oracle, one thread", "seconds_per_step": t}
    return out


def run_reference_dg(args):
    t, nnz = dg_cpu_sample(DGSYS["cpu_n"], args.seed)
    v = nnz / t
    return {"impl": "reference", "metric": "matrix nnz/s (DG1 interior penalty)", "value": v, "unit": "nnz/s",
            "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": DGSYS["desc"], "sample_n": DGSYS["cpu_n"], "nnz": nnz},
            "cpu_baseline": {"value": v, "unit": "nnz/s", "cores": 1, "kind": "port",
                             "sample": f"n={DGSYS['cpu_n']} DG1 system, numpy oracle (the reference needs DOLFINx)"},
            "e2e": {"value": v, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def multimesh_inputs(seed: int):
    rng = np.random.default_rng(seed)
    ns = rng.integers(MULTI["nmin"], MULTI["nmax"] + 1, size=MULTI["count"])
    kinds = rng.permutation(["p1", "p2"] * (MULTI["count"] // 2))
    return [make_inputs(str(k), int(n), seed=seed + i, precision="fp32" if k == "p2" else "fp64")
            for i, (k, n) in enumerate(zip(kinds, ns))]


def run_gpu_multimesh(args, rank, world, local_rank):
    import torch

    import cudolfinx as cx
    from cudolfinx import _lib

    torch.cuda.set_device(local_rank)
    t_setup = time.perf_counter()
    Is = multimesh_inputs(args.seed)
    asm = cx.CUDAAssembler()
    items = []
    for I in Is:
        a = cx.form(I["a"])
        items.append((a, asm.create_matrix(a), asm.pack_bcs([I["bc"]])))
    t_tune = time.perf_counter()
    G = cx.AssemblyGraph(items, variants="tune", branches=args.graph_branches)
    tune_s = time.perf_counter() - t_tune
    G.capture()
    setup_s = time.perf_counter() - t_setup
    nnz = G.nnz
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        G.replay()
    torch.cuda.synchronize()
    dist = torch.distributed if world > 1 else None
    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed launches (--nvtx-include timed/)
    e0.record(stream)
    for _ in range(args.steps):
        G.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    total_ms = e0.elapsed_time(e1)
    clk = clocks.stop()

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(reps):
            fn()
        a1.record(stream)
        torch.cuda.synchronize()
        return a0.elapsed_time(a1) / reps

    eager_ms = timed(G.run_eager, max(1, args.steps // 2))
    # plain path: one call per mesh, engine default variant, FP64 element tensors
    from cudolfinx import fem

    fp64_items = []
    for I, (a, mat, bcs) in zip(Is, items):
        if I["kind"] == "p2":
            a64 = cx.form(fem.stiffness(I["V"], I["a"].coefficients[0]))
            fp64_items.append((a64, cx.CUDAMatrix(asm._ctx, mat.sparsity), bcs))
        else:
            fp64_items.append((a, mat, bcs))
    plain = cx.AssemblyGraph(fp64_items, variants="auto")
    plain_ms = timed(plain.run_eager, max(1, args.steps // 2))
    total_ms, eager_ms, plain_ms = reduce_over_ranks([total_ms, eager_ms, plain_ms])
    ms = total_ms / args.steps
    alg = sum(algorithmic_matrix_bytes(I, it[1].sparsity.nnz) for I, it in zip(Is, items))
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg / (ms / 1e3) / 1e9
    launches = sum(matrix_kernels(I["kind"], it["variant"], len(I["cells"]) >= (1 << 20), item[1].sparsity.nnz)
                   for I, item, it in zip(Is, items, G.items))
    chosen = {}
    for it in G.items:
        chosen[it["variant"]] = chosen.get(it["variant"], 0) + 1
    out = {
        "metric": "matrix nnz/s (multi-mesh graph)",
        "value": replica_rate(nnz, args.steps, total_ms, world),
        "unit": "nnz/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-element(P2)/f64-accumulate",
        "data": "synthetic (seeded numpy inputs)",
        "config": {"workload": MULTI["desc"], "meshes": len(Is), "cells": sum(len(I["cells"]) for I in Is),
                   "nnz": nnz, "ns": [int(I["n"]) for I in Is], "kinds": [I["kind"] for I in Is],
                   "variants_chosen": chosen, "step": "one CUDA graph replay: every mesh's matrix assembly "
                   "(zero, assemble with BC skip, unit diagonal)", "graph_branches": args.graph_branches,
                   "l2": "inputs larger than L2",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "kernel": "graph of matrix assemblies", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": None, "algorithmic_bytes": alg,
                     "kernel_ms": ms, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"
                     if "hbm_gbs" in peaks else "fallback 6650 GB/s"},
        "eager_same_variants_ms": eager_ms,
        "plain_fp64": {"ms": plain_ms, "path": "one fe_assemble_matrix per mesh, default variant, FP64 element "
                       "tensors, no graph", "speedup_of_graph": plain_ms / ms},
        "gpu_launches": launches * args.steps,
        "clocks": clk, "setup_s": setup_s, "tune_s": tune_s,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import cfem

        threads = os.cpu_count() or 1
        sample = list(range(0, len(Is), MULTI["cpu_every"]))
        tsum, nsum = 0.0, 0
        for i in sample:
            rp, cl = items[i][1].sparsity.to_host()
            Cq = cfem.CpuAssembler(oracle_problem(Is[i]), rp, cl, nthreads=threads)
            Cq.assemble_matrix()
            t0 = time.perf_counter()
            Cq.assemble_matrix()
            tsum += time.perf_counter() - t0
            nsum += len(cl)
            Cq.close()
        out["cpu_baseline"] = {"value": nsum / tsum, "unit": "nnz/s", "cores": threads, "kind": "port",
                               "sample": f"matrix assembly of meshes {sample} (every {MULTI['cpu_every']}th), "
                                         f"{threads} threads, C port of the reference CPU path (oracle/cfem.c)"}
    return out


def run_reference_multimesh(args):
    from oracle import cfem

    Is = multimesh_inputs(args.seed)
    sample = list(range(0, len(Is), MULTI["cpu_every"]))
    threads = os.cpu_count() or 1
    asms = []
    nnz = 0
    for i in sample:
        rp, cl = host_pattern(Is[i])
        asms.append(cfem.CpuAssembler(oracle_problem(Is[i]), rp, cl, nthreads=threads))
        nnz += len(cl)

    def one_step():
        t0 = time.perf_counter()
        for Cq in asms:
            Cq.assemble_matrix()
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        one_step()
    times = [one_step() for _ in range(args.steps)]
    for Cq in asms:
        Cq.close()
    total = sum(times)
    v = nnz * args.steps / total
    return {"impl": "reference", "metric": "matrix nnz/s (multi-mesh graph)", "value": v, "unit": "nnz/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": MULTI["desc"], "meshes_timed": sample, "nnz": nnz,
                       "step": "matrix assembly of every %dth mesh (bounded sample)" % MULTI["cpu_every"]},
            "cpu_baseline": {"value": v, "unit": "nnz/s", "cores": threads, "kind": "port",
                             "sample": f"meshes {sample}; C port of the reference CPU path (oracle/cfem.c)"},
            "e2e": {"value": v, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def serve_request_bytes(kind, n, iterations, solver="fp64"):
    """Bytes one request must move: its matrix assembly (values written,
    slot map, dofmap, geometry, coordinates, coefficients), b, and per PCG
    iteration one SpMV (values and columns: 12 B per entry in FP64; 4 + 4/9 B
    in the FP32 3x3 block-column layout the server's mixed solver uses for
    vector P2; row pointers, p, Ap) plus the vector updates (x, r, z, p, Ap,
    dinv).  For vector P2 with solver="mixed" the iterations are the FP32
    inner ones; the FP64 refinement passes (a few per request) are not
    counted."""
    from cudolfinx import serve

    sz = serve.problem_sizes(kind, n)
    C, N, nnz, k = sz["cells"], sz["rows"], sz["nnz"], sz["k"]
    asm = 8 * nnz + k * k * C + 4 * k * C + 16 * C + 24 * sz["vertices"] + 8 * C * (2 if kind == "vp2" else 1)
    vec = 8 * N + 4 * k * C + 16 * C
    # the server's mixed solver runs FP32 inner iterations for vector P2 only
    per_nnz = 4 + 4 / 9 if (solver == "mixed" and kind == "vp2") else 12
    per_it = per_nnz * nnz + 4 * N + 16 * N + 8 * 10 * N
    return asm + vec + iterations * per_it


def serve_working_set(kind, n, solver="fp64"):
    """Bytes a request's PCG iterations touch again and again (matrix values
    and columns, row pointers, six vectors): below the 126 MB L2 they stay
    in L2 from one iteration to the next."""
    from cudolfinx import serve

    sz = serve.problem_sizes(kind, n)
    per_nnz = 4 + 4 / 9 if (solver == "mixed" and kind == "vp2") else 12
    return per_nnz * sz["nnz"] + (4 + 6 * 8) * sz["rows"]


def serve_launches(iterations):
    # matrix (zero, kernel, diagonal) + right-hand side (zero, lifting, vector with set_bc) + PCG (2 + 80 per 16
    # iterations)
    return 3 + 3 + 2 + 80 * ((iterations + 16) // 16)


def run_gpu_serve(args, rank, world, local_rank):
    import torch

    from cudolfinx import serve

    torch.cuda.set_device(local_rank)
    count = args.serve_requests or SERVE["requests"]
    rates = [float(r) for r in (args.serve_rates.split(",") if args.serve_rates else SERVE["rates"])]
    nmax = args.serve_nmax or SERVE["nmax"]
    seed = args.seed + 7919 * rank
    t_setup = time.perf_counter()
    base = serve.make_requests(count, rates[0], seed=seed, nmin=SERVE["nmin"], nmax=nmax)
    if args.serve_workers:
        SERVE["workers"] = args.serve_workers
    srv = serve.Server(workers=SERVE["workers"], hbm_budget=SERVE["budget_gb"] << 30, precision="fp32")
    keys = sorted({r.key for r in base})
    srv.warm(keys)
    setup_s = time.perf_counter() - t_setup
    # warm-up: a few requests through the running server
    srv.run(serve.make_requests(4, 0.0, seed=seed + 1, nmin=SERVE["nmin"], nmax=min(nmax, 16)))
    clocks = ClockSampler(local_rank)
    clocks.start()
    per_rate = []
    served_results = None
    for rate in rates:
        reqs = serve.make_requests(count, rate, seed=seed, nmin=SERVE["nmin"], nmax=nmax)
        res = srv.run(reqs)
        summ = serve.summarize(res)
        summ["rate_rps"] = rate
        per_rate.append(summ)
        served_results = res
    clk = clocks.stop()
    # plain path: one request at a time, FP64, nothing cached, same requests at the lowest rate
    plain_res = serve.Server(plain=True).run(serve.make_requests(count, rates[0], seed=seed, nmin=SERVE["nmin"],
                                                                 nmax=nmax))
    plain = serve.summarize(plain_res)
    plain["rate_rps"] = rates[0]
    diffs = [serve.solution_difference(a, b) for a, b in zip(served_results, plain_res)]
    # precision: a subset solved to rtol 1e-12 with FP64 and FP32 element
    # tensors, so the difference is the discretisation's and not where two
    # PCG runs stop; the served rtol-1e-8 results are compared with it too
    import dataclasses

    sub = base[:min(len(base), 12)]
    tight = [dataclasses.replace(r, rtol=1e-12) for r in sub]
    ref64 = serve.Server(workers=SERVE["workers"], precision="fp64", solver="fp64").run(tight)
    t32 = serve.Server(workers=SERVE["workers"], precision="fp32", solver=srv.solver).run(tight)
    prec = {}
    for fam in serve.FAMILIES:
        idx = [i for i, r in enumerate(sub) if r.kind == fam]
        if not idx:
            continue
        prec[fam] = {"requests": len(idx), "n": [sub[i].n for i in idx],
                     "served_precision_vs_fp64_at_rtol_1e-12": max(serve.solution_difference(t32[i], ref64[i])
                                                                   for i in idx),
                     "served_rtol_1e-8_vs_fp64_at_rtol_1e-12": max(serve.solution_difference(served_results[i],
                                                                                             ref64[i])
                                                                   for i in idx),
                     "plain_rtol_1e-8_vs_fp64_at_rtol_1e-12": max(serve.solution_difference(plain_res[i], ref64[i])
                                                                  for i in idx)}
    top = per_rate[-1]
    done = [r for r in served_results if r.error is None]
    alg = sum(serve_request_bytes(r.kind, r.n, r.iterations, srv.solver) for r in done)
    l2_alg = sum(serve_request_bytes(r.kind, r.n, r.iterations, srv.solver) for r in done
                 if serve_working_set(r.kind, r.n, srv.solver) < L2_BYTES)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg / top["makespan_s"] / 1e9
    value = top["throughput_rps"]
    (value,) = reduce_over_ranks([value], op="min")
    value *= world
    out = {
        "metric": "served assemble+solve requests/s (p50/p99 latency beside)",
        "value": value, "unit": "req/s", "n_gpus": world, "steps": count, "warmup": 4,
        "ms_per_step": 1e3 / top["throughput_rps"] if top["throughput_rps"] else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-element(P2, vP2)/f64-accumulate; PCG f32-inner/f64-refined (vP2), f64 (P1, P2)",
        "data": "synthetic (seeded request stream)",
        "config": {"workload": SERVE["desc"] + f" in [{SERVE['nmin']}, {nmax}] (bounded sample of the "
                   f"10,000-request stream: {count} requests per rate)", "requests": count, "rates_rps": rates,
                   "workers": SERVE["workers"], "hbm_budget_gb": SERVE["budget_gb"],
                   "cache": f"warm: one slot per (family, n) of the stream built before the timed runs "
                            f"({len(keys)} sizes)",
                   "step": "one request: H2D coefficients, assemble A and b (lifting, set_bc), PCG, D2H x",
                   "parallelism": f"replicas x{world}"},
        "latency": {"per_rate": per_rate, "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"]},
        "plain_fp64": {**plain, "path": "one request at a time, FP64 element tensors, mesh/pattern/forms built "
                                        "per request", "speedup_of_served": (top["throughput_rps"] /
                                                                             plain["throughput_rps"])
                       if plain["throughput_rps"] else None},
        "precision": {"note": "served_precision_vs_fp64_at_rtol_1e-12: the served path (FP32 element tensors of P2 "
                              "and vector-P2, FP32 inner PCG with FP64 refinement) against FP64 throughout, both "
                              "solved to rtol 1e-12, so the difference is the precision's alone (the <= 1e-6 "
                              "bound); the rtol-1e-8 rows add where each PCG run stops, for the served and the "
                              "plain FP64 path alike",
                      "served_vs_plain_max_rel_diff": max(diffs) if diffs else None,
                      "served_vs_plain_median_rel_diff": float(np.median(diffs)) if diffs else None,
                      "per_family": prec},
        "roofline": {"bound": "hbm", "kernel": "served request mix (assembly + PCG)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "algorithmic_bytes": alg, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"
                     if "hbm_gbs" in peaks else "fallback 6650 GB/s",
                     "l2_resident_share": l2_alg / alg if alg else None,
                     "note": "bytes of the requests whose PCG working set (values, columns, vectors) fits in the "
                             "126 MB L2 are served from L2 on every iteration after the first; that share "
                             "(l2_resident_share) can lift the fraction of HBM above 1"},
        "gpu_launches": sum(serve_launches(r.iterations) for r in served_results if r.error is None),
        "e2e": {"value": top["throughput_rps"], "unit": "req/s",
                "h2d_bytes_per_step": int(np.mean([8 * sum(c.size for c in r.coef) for r in base])),
                "d2h_bytes_per_step": int(np.mean([8 * serve.problem_sizes(r.kind, r.n)["rows"] for r in base])),
                "note": "every request is end to end: host coefficients in, solution out"},
        "clocks": clk, "setup_s": setup_s, "max_concurrent": srv.max_concurrent,
        "ledger_peak_gb": srv.ledger.peak / 2 ** 30,
    }
    return out


def run_reference_serve(args):
    """C port of the reference CPU path on a bounded sample of the request
    stream: assembly only (the reference hands the system to PETSc KSP, which
    is not part of this build), one request at a time."""
    from oracle import cfem
    from cudolfinx import serve

    count = min(args.serve_requests or SERVE["requests"], 24)
    nmax = args.serve_nmax or SERVE["nmax"]
    reqs = serve.make_requests(count, 0.0, seed=args.seed, nmin=SERVE["nmin"], nmax=nmax)
    threads = os.cpu_count() or 1
    t_all = 0.0
    for r in reqs:
        kind = {"p1": "p1", "p2": "p2", "vp2": "vp2"}[r.kind]
        I = make_inputs(kind, r.n, seed=args.seed)
        rp, cl = host_pattern(I)
        P = oracle_problem(I)
        if kind == "vp2":
            P["lam"], P["mu"] = r.coef
        elif kind == "p1":
            P["kind"] = "p1k"
            P["k"] = r.coef[0]
        Cq = cfem.CpuAssembler(P, rp, cl, nthreads=threads)
        t0 = time.perf_counter()
        Cq.assemble_matrix()
        Cq.assemble_rhs()
        t_all += time.perf_counter() - t0
        Cq.close()
    v = count / t_all
    return {"impl": "reference", "metric": "served assemble+solve requests/s (p50/p99 latency beside)", "value": v,
            "unit": "req/s", "n_gpus": 1, "steps": count, "warmup": 0, "ms_per_step": 1e3 * t_all / count,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded request stream)",
            "config": {"workload": SERVE["desc"], "requests_timed": count,
                       "step": "assembly of A and b (lifting, set_bc) per request; solve not included"},
            "cpu_baseline": {"value": v, "unit": "req/s", "cores": threads, "kind": "port",
                             "sample": f"{count} requests, assembly only, C port of the reference CPU path"},
            "e2e": {"value": v, "unit": "req/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference(args):
    if args.workload == "serve":
        return run_reference_serve(args)
    if args.workload == "batch":
        return run_reference_batch(args)
    if args.workload == "multimesh":
        return run_reference_multimesh(args)
    if args.workload == "blocksys":
        return run_reference_blocksys(args)
    if args.workload == "interp":
        return run_reference_interp(args)
    if args.workload == "dg":
        return run_reference_dg(args)
    # the CPU path alone: problem, pattern and assembly from oracle/ (numpy
    # builders + the C restatement); nothing of the engine is loaded
    from oracle import cfem
    from oracle import fem_oracle as fo

    W = WORKLOADS[args.workload]
    P = fo.build_problem(W["kind"], W["n"], seed=args.seed)
    threads = os.cpu_count() or 1
    row_ptr, col = cfem.pattern(P["dofs"], P["ndof"], P["bs"], nthreads=threads)
    nnz = len(col)
    C = cfem.CpuAssembler(P, row_ptr, col, nthreads=threads)
    for _ in range(args.warmup):
        cpu_step(C)
    times = [cpu_step(C) for _ in range(args.steps)]
    C.close()
    total = sum(times)
    v = nnz * args.steps / total
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {"impl": "reference", "metric": "matrix nnz/s", "value": v, "unit": "nnz/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded numpy inputs with the configuration's shapes and distributions)",
            "config": workload_config(W, len(P["cells"]), P["ndof"] * P["bs"], nnz, world),
            "cpu_baseline": {"value": v, "unit": "nnz/s", "cores": threads, "kind": "port",
                             "sample": "full workload each step; C port of the reference CPU path "
                                       "(oracle/cfem.c); the reference itself needs DOLFINx + PETSc"},
            "e2e": {"value": v, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference_batch(args):
    import torch

    I = batch_inputs(args.seed)
    row_ptr, col = host_pattern(I)
    nnz = len(col)
    kd = batch_coefficients(BATCH["cpu_sample"], len(I["cells"]), args.seed + 1000, "cpu")
    from oracle import cfem

    threads = os.cpu_count() or 1
    P = oracle_problem(I)
    P["kind"] = "p1k"
    P["k"] = kd[0].numpy()
    Cq = cfem.CpuAssembler(P, row_ptr, col, nthreads=threads)

    def one_step():
        t0 = time.perf_counter()
        for s in range(BATCH["cpu_sample"]):
            Cq.c0 = np.ascontiguousarray(kd[s].numpy())
            Cq.assemble_matrix()
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        one_step()
    times = [one_step() for _ in range(args.steps)]
    Cq.close()
    total = sum(times)
    v = nnz * BATCH["cpu_sample"] * args.steps / total
    del torch
    return {"impl": "reference", "metric": "matrix nnz/s (batched instances)", "value": v, "unit": "nnz/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": BATCH["desc"], "cells": len(I["cells"]), "nnz": nnz,
                       "step": f"{BATCH['cpu_sample']} instances (bounded sample), one assembly each"},
            "cpu_baseline": {"value": v, "unit": "nnz/s", "cores": threads, "kind": "port",
                             "sample": f"{BATCH['cpu_sample']} instances per step; C port of the reference CPU "
                                       "path (oracle/cfem.c), which has no batch path"},
            "e2e": {"value": v, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batch", "multimesh", "serve", "blocksys", "interp", "dg"],
                    default="p2")
    ap.add_argument("--variant", choices=["auto", "tile", "atomic", "atomic-full", "sorted-slot", "deterministic",
                                          "row-gather", "block", "grouped", "coalesced"], default="auto")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--graph-branches", type=int, default=8,
                    help="multimesh: parallel branches of the captured graph (independent meshes overlap)")
    ap.add_argument("--serve-requests", type=int, default=0, help="serve workload: requests per rate")
    ap.add_argument("--serve-rates", default="", help="serve workload: comma-separated arrival rates (req/s)")
    ap.add_argument("--serve-nmax", type=int, default=0, help="serve workload: largest n (default 48)")
    ap.add_argument("--serve-workers", type=int, default=0, help="serve workload: worker streams (default 4)")
    ap.add_argument("--instances", type=int, default=0,
                    help="batch workload: number of instances (default 256; smaller for profiling)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="time eager steps instead of replaying a CUDA graph")
    ap.add_argument("--launch", default="", help="launch shape of the P1/P2 scatter: CELLS_PER_CTA,STAGE "
                    "(fe_form_set_launch; e.g. 64,0)")
    ap.add_argument("--rhs", choices=["fused", "calls"], default="fused",
                    help="right-hand side of the step: fe_assemble_rhs (default) or the three calls "
                         "(assemble_vector, apply_lifting, set_bc)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the full-size parity check against the oracle")
    ap.add_argument("--no-precision", action="store_true", help="skip the FP32-vs-FP64 precision report")
    ap.add_argument("--precision-rtol", type=float, default=1e-10,
                    help="PCG tolerance of the precision report's two solves")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        runner = {"batch": run_gpu_batch, "multimesh": run_gpu_multimesh, "serve": run_gpu_serve,
                  "blocksys": run_gpu_blocksys, "interp": run_gpu_interp,
                  "dg": run_gpu_dg}.get(args.workload, run_gpu)
        out = runner(args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
