"""Generate the golden fixtures in this directory from the numpy oracle.

    python tests/golden/make_golden.py

The reference ships no golden vectors (its tests compare against DOLFINx at
run time, python/test/test_cuda_assembly.py:93-209) and DOLFINx cannot run in
this environment, so these fixtures freeze the oracle's output on small
meshes: mesh, dofmap, BC dofs, coefficients, CSR pattern, assembled matrix
(BCs applied, unit diagonal) and right-hand side (vector + lifting + set_bc),
and each entry's parity bound (A_bound, b_bound: fem_oracle.matrix_bound,
vector_bound + lifting_bound, 0 where set_diagonal / set_bc write).
They pin the oracle against regressions and give the GPU tests inputs that do
not depend on the generators.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import fem_oracle as fo  # noqa: E402

CASES = [("p1", 2), ("p1", 3), ("p1k", 2), ("p2", 2), ("vp2", 2), ("p3", 2)]


def make(kind, n):
    P = fo.build_problem(kind, n, seed=0)
    S = fo.solve_system(P)
    out = dict(coords=P["coords"], cells=P["cells"], dofs=P["dofs"], bc_dofs=P["bc_dofs"],
               row_ptr=S["row_ptr"], col=S["col"], A=S["A"], b=S["b"], g=P["g"],
               A_bound=S["A_bound"], b_bound=S["b_bound"],
               ndof=np.array(P["ndof"]), bs=np.array(P["bs"]), n=np.array(n))
    for key in ("k", "f", "lam", "mu"):
        if P.get(key) is not None:
            out[key] = np.asarray(P[key])
    return out


def main():
    for kind, n in CASES:
        np.savez_compressed(os.path.join(HERE, f"{kind}_n{n}.npz"), **make(kind, n))


if __name__ == "__main__":
    main()
