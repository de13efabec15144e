"""Helpers shared by the GPU tests: build a problem through the cudolfinx
mirror API (C-ABI underneath) from the oracle's inputs, and compare."""
import numpy as np

from conftest import ensure_library


def tolerance_check(gpu, ref, bound):
    """Entrywise |gpu - ref| <= bound, the oracle's per-entry parity bound
    (fem_oracle.matrix_bound / vector_bound / lifting_bound: 1e-12 times the
    sum of the entry's |contributions| plus 1e-14 times each contributing
    element's largest |entry|; 0 where the value is written, not summed).
    Returns (ok, worst |gpu - ref| / bound)."""
    from oracle import fem_oracle as fo

    return fo.within_bound(gpu, ref, bound)


def mirror_problem(P, precision="fp64"):
    """Mesh/spaces/forms/BC through the mirror API for an oracle problem P."""
    ensure_library()
    import cudolfinx as cx
    from cudolfinx import fem

    mesh = fem.Mesh(P["coords"], P["cells"], grid_n=P["n"])
    kind = P["kind"]
    out = {"mesh": mesh}
    if kind in ("p1", "p1k"):
        V = fem.functionspace(mesh, ("P", 1))
        assert np.array_equal(V.dofs, P["dofs"])
        if kind == "p1":
            k = 1.0
        else:
            W = fem.functionspace(mesh, ("DG", 0))
            k = fem.Function(W, P["k"])
        fP1 = fem.Function(V, P["f"])
        a = fem.stiffness(V, k)
        L = fem.load(V, fP1)
    elif kind == "p2":
        V = fem.functionspace(mesh, ("P", 2))
        assert np.array_equal(V.dofs, P["dofs"])
        V1 = fem.functionspace(mesh, ("P", 1))
        W = fem.functionspace(mesh, ("DG", 0))
        a = fem.stiffness(V, fem.Function(V1, P["k"]), precision=precision)
        L = fem.load(V, fem.Function(W, P["f"]))
    elif kind == "p3":
        V = fem.functionspace(mesh, ("P", 3))
        assert np.array_equal(V.dofs, P["dofs"])
        W = fem.functionspace(mesh, ("DG", 0))
        a = fem.stiffness(V, fem.Function(W, P["k"]), precision=precision)
        L = fem.load(V, fem.Function(W, P["f"]))
    elif kind == "vp2":
        V = fem.functionspace(mesh, ("P", 2, (3,)))
        W = fem.functionspace(mesh, ("DG", 0))
        a = fem.elasticity(V, fem.Function(W, P["lam"]), fem.Function(W, P["mu"]), precision=precision)
        W3 = fem.functionspace(mesh, ("DG", 0, (3,)))
        L = fem.load(V, fem.Function(W3, np.asarray(P["f"]).reshape(-1)))
    else:
        raise ValueError(kind)
    g = fem.Function(V, P["g"])
    bc = fem.dirichletbc(g, P["bc_dofs"])
    out.update(V=V, a=a, L=L, bc=bc)
    out["cx"] = cx
    return out


def run_system(P, deterministic=False, precision="fp64", variant="auto"):
    """A (host CSR arrays) and b through the mirror API: assemble_matrix with
    BCs, assemble_vector + apply_lifting + set_bc."""
    M = mirror_problem(P, precision)
    cx = M["cx"]
    asm = cx.CUDAAssembler()
    a = cx.form(M["a"])
    L = cx.form(M["L"])
    bcs = asm.pack_bcs([M["bc"]])
    A = asm.assemble_matrix(a, bcs=bcs, deterministic=deterministic, variant=variant)
    A.assemble()
    b = asm.assemble_vector(L)
    asm.apply_lifting(b, [a], [bcs])
    asm.set_bc(b, bcs, M["V"])
    rp, col = A.sparsity.to_host()
    return {"row_ptr": rp, "col": col, "A": A.values.cpu().numpy(), "b": b.to_host(), "asm": asm, "Aobj": A,
            "bobj": b, "forms": (a, L), "bcs": bcs, "M": M}
