"""Build-time generator of the element-tensor bodies used by the CUDA kernels.

The reference wraps FFCx ``tabulate_tensor`` C bodies into NVRTC kernels at
run time (python/cudolfinx/jit.py:61-114, cpp/cudolfinx/fem/CUDAFormIntegral.cpp:
2366-2469).  For the built-in forms this engine writes the element tensors
from the mathematics instead: the reference-element tensors below are
integrated exactly in rational arithmetic and emitted as straight-line
``fma`` code with every structurally-zero term removed (744 of 1320 terms
survive for P2 stiffness with a P1 coefficient).

Output: fe_element_code.cuh (regenerated by the package build when this file
is newer).

Conventions
* P2 local dofs: 4 vertices, then edges in basix order (2,3),(1,3),(1,2),(0,3),(0,2),(0,1).
* Symmetric geometry pairs s: (0,0),(1,1),(2,2),(0,1),(0,2),(1,2).
* Unique symmetric entries e enumerate (i, j) with i <= j row by row.
"""
from __future__ import annotations

import os
import sys
from fractions import Fraction
from math import factorial

EDGES = ((2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1))
PAIRS = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))


def mono_int(a, b, c):
    return Fraction(factorial(a) * factorial(b) * factorial(c), factorial(a + b + c + 3))


def pmul(p, q):
    r = {}
    for k1, v1 in p.items():
        for k2, v2 in q.items():
            k = (k1[0] + k2[0], k1[1] + k2[1], k1[2] + k2[2])
            r[k] = r.get(k, 0) + v1 * v2
    return {k: v for k, v in r.items() if v != 0}


def padd(p, q, s=1):
    r = dict(p)
    for k, v in q.items():
        r[k] = r.get(k, 0) + s * v
    return {k: v for k, v in r.items() if v != 0}


def pdiff(p, ax):
    r = {}
    for k, v in p.items():
        if k[ax]:
            kk = list(k)
            kk[ax] -= 1
            r[tuple(kk)] = r.get(tuple(kk), 0) + v * k[ax]
    return r


def pint(p):
    return sum((v * mono_int(*k) for k, v in p.items()), Fraction(0))


LAM = [
    {(0, 0, 0): Fraction(1), (1, 0, 0): Fraction(-1), (0, 1, 0): Fraction(-1), (0, 0, 1): Fraction(-1)},
    {(1, 0, 0): Fraction(1)},
    {(0, 1, 0): Fraction(1)},
    {(0, 0, 1): Fraction(1)},
]
PHI = ([pmul(l, padd({k: 2 * v for k, v in l.items()}, {(0, 0, 0): Fraction(1)}, -1)) for l in LAM]
       + [{k: 4 * v for k, v in pmul(LAM[a], LAM[b]).items()} for a, b in EDGES])
DPHI = [[pdiff(p, ax) for ax in range(3)] for p in PHI]
UNIQ = [(i, j) for i in range(10) for j in range(i, 10)]


def _scale(p, c):
    return {k: c * v for k, v in p.items()}


def _const(c):
    return {(0, 0, 0): Fraction(c)}


# P3 Lagrange, equispaced points (basix's "equispaced" variant): vertices,
# then two dofs per edge in the basix edge order (the point nearer the edge's
# first vertex first), then one dof per face (face f opposite vertex f)
FACES = ((1, 2, 3), (0, 2, 3), (0, 1, 3), (0, 1, 2))
PHI3 = ([_scale(pmul(l, pmul(padd(_scale(l, 3), _const(1), -1), padd(_scale(l, 3), _const(2), -1))),
                Fraction(1, 2)) for l in LAM]
        + [q for a, b in EDGES
           for q in (_scale(pmul(pmul(LAM[a], LAM[b]), padd(_scale(LAM[a], 3), _const(1), -1)), Fraction(9, 2)),
                     _scale(pmul(pmul(LAM[a], LAM[b]), padd(_scale(LAM[b], 3), _const(1), -1)), Fraction(9, 2)))]
        + [_scale(pmul(pmul(LAM[a], LAM[b]), LAM[c]), 27) for a, b, c in FACES])
DPHI3 = [[pdiff(p, ax) for ax in range(3)] for p in PHI3]
UNIQ3 = [(i, j) for i in range(20) for j in range(i, 20)]


def r3_plain(a, b, i, j):
    return pint(pmul(DPHI3[i][a], DPHI3[j][b]))


def lit(x: Fraction) -> str:
    """Exact-as-possible C double literal (hex float of the rounded value)."""
    return float(x).hex()


def sum_expr(var, terms, chains=4):
    """sum_t var[idx_t] * c_t as up to `chains` independent fma chains added
    by a balanced tree: the critical path is ~len/chains fmas instead of len."""
    if not terms:
        return "T(0)"
    n = min(chains, len(terms))
    parts = []
    for k in range(n):
        sub = terms[k::n]
        idx, c = sub[0]
        e = f"{var}[{idx}] * T({lit(c)})"
        for idx, c in sub[1:]:
            e = f"fma({var}[{idx}], T({lit(c)}), {e})"
        parts.append(e)
    while len(parts) > 1:
        parts = [f"({parts[q]} + {parts[q + 1]})" if q + 1 < len(parts) else parts[q]
                 for q in range(0, len(parts), 2)]
    return parts[0]


def symmetric_body(exprs, n):
    """Body emitting the unique entries i <= j of a symmetric element block.

    FP64: every entry from its expression.  FP32: the off-diagonal entries
    from their expressions (in T), each diagonal entry as minus the FP64 sum
    of the row's off-diagonal entries.  The exact block has zero row sums
    (the basis sums to one), and keeping them exact after FP32 rounding stops
    the rounding from acting on the smooth, badly conditioned modes: on P2
    Poisson the solution error of FP32 element tensors drops by about three
    orders of magnitude at the same matrix error."""
    out = ["  if constexpr (sizeof(T) == 8) {\n"]
    for (i, j), e in exprs.items():
        out.append(f"    emit({i}, {j}, {e});\n")
    out.append("  } else {\n")
    out.append(f"    double rs[{n}] = {{{', '.join(['0.0'] * n)}}};\n")
    for (i, j), e in exprs.items():
        if i != j:
            out.append(f"    {{ const T v = {e}; rs[{i}] += (double)v; rs[{j}] += (double)v; emit({i}, {j}, v); }}\n")
    for i in range(n):
        out.append(f"    emit({i}, {i}, -rs[{i}]);\n")
    out.append("  }\n")
    return "".join(out)


def full_body(exprs, n):
    """Body emitting all entries of a coupling block between two displacement
    components.  FP32: off-diagonal entries in T, each diagonal entry as minus
    the mean of the FP64 row and column sums of the off-diagonal entries (the
    exact block has zero row and column sums; the block's transpose is emitted
    with the same values, so the mean keeps the element matrix symmetric)."""
    out = ["  if constexpr (sizeof(T) == 8) {\n"]
    for (i, j), e in exprs.items():
        out.append(f"    emit({i}, {j}, {e});\n")
    out.append("  } else {\n")
    out.append(f"    double rs[{n}] = {{{', '.join(['0.0'] * n)}}};\n")
    out.append(f"    double cs[{n}] = {{{', '.join(['0.0'] * n)}}};\n")
    for (i, j), e in exprs.items():
        if i != j:
            out.append(f"    {{ const T v = {e}; rs[{i}] += (double)v; cs[{j}] += (double)v; emit({i}, {j}, v); }}\n")
    for i in range(n):
        out.append(f"    emit({i}, {i}, -0.5 * (rs[{i}] + cs[{i}]));\n")
    out.append("  }\n")
    return "".join(out)


def r_weighted(m, a, b, i, j):
    return pint(pmul(LAM[m], pmul(DPHI[i][a], DPHI[j][b])))


def r_plain(a, b, i, j):
    return pint(pmul(DPHI[i][a], DPHI[j][b]))


def sym_pair(fn, s, i, j):
    a, b = PAIRS[s]
    v = fn(a, b, i, j)
    if a != b:
        v += fn(b, a, i, j)
    return v


FACETS = ((1, 2, 3), (0, 2, 3), (0, 1, 3), (0, 1, 2))  # facet f opposite vertex f


def bary_basis(degree):
    """Basis functions as polynomials in the four barycentric coordinates."""
    lam = [{tuple(1 if q == m else 0 for q in range(4)): Fraction(1)} for m in range(4)]

    def mul(p, q):
        r = {}
        for k1, v1 in p.items():
            for k2, v2 in q.items():
                k = tuple(a + b for a, b in zip(k1, k2))
                r[k] = r.get(k, 0) + v1 * v2
        return {k: v for k, v in r.items() if v != 0}

    if degree == 1:
        return lam, lam, mul
    vert = []
    for m in range(4):
        p = {k: 2 * v for k, v in mul(lam[m], lam[m]).items()}
        for k, v in lam[m].items():
            p[k] = p.get(k, 0) - v
        vert.append(p)
    edge = [{k: 4 * v for k, v in mul(lam[a], lam[b]).items()} for a, b in EDGES]
    return vert + edge, lam, mul


def bary_facet_int(p, f):
    """int_F p / |F| for p in barycentric monomials: 2 a! b! c! / (a+b+c+2)!,
    lambda_f = 0 on facet f."""
    tot = Fraction(0)
    for k, v in p.items():
        if k[f]:
            continue
        e = [k[m] for m in range(4) if m != f]
        tot += v * Fraction(2 * factorial(e[0]) * factorial(e[1]) * factorial(e[2]), factorial(sum(e) + 2))
    return tot


def facet_tables() -> str:
    """Exterior-facet reference tensors, per local facet f, over the cell-local
    dofs that lie on f (the others vanish there): mass int phi_i phi_j / |F|,
    load int phi_i / |F| and P1-weighted load int lambda_m phi_i / |F|.
    Compiled only where FE_FACET_TABLES is defined."""
    out = ["#ifdef FE_FACET_TABLES\n"]
    for degree in (1, 2):
        phi, lam, mul = bary_basis(degree)
        k = len(phi)
        on = []
        for f in range(4):
            verts = [v for v in range(4) if v != f]
            dofs = list(verts)
            if degree == 2:
                dofs += [4 + e for e, (a, b) in enumerate(EDGES) if f not in (a, b)]
            on.append(dofs)
        nd = len(on[0])
        P = f"P{degree}"
        out.append(f"// cell-local dofs on each facet ({P})\n")
        out.append(f"static __constant__ int kFacetDofs{P}[4][{nd}] = {{" +
                   ", ".join("{" + ", ".join(str(d) for d in on[f]) + "}" for f in range(4)) + "};\n")
        mass = [[[bary_facet_int(mul(phi[on[f][a]], phi[on[f][b]]), f) for b in range(nd)] for a in range(nd)]
                for f in range(4)]
        load = [[bary_facet_int(phi[on[f][a]], f) for a in range(nd)] for f in range(4)]
        wl = [[[bary_facet_int(mul(lam[m], phi[on[f][a]]), f) for a in range(nd)] for m in range(4)]
              for f in range(4)]
        out.append(f"static __constant__ double kFacetMass{P}[4][{nd}][{nd}] = {{" +
                   ", ".join("{" + ", ".join("{" + ", ".join(lit(x) for x in row) + "}" for row in mass[f]) + "}"
                             for f in range(4)) + "};\n")
        out.append(f"static __constant__ double kFacetLoad{P}[4][{nd}] = {{" +
                   ", ".join("{" + ", ".join(lit(x) for x in load[f]) + "}" for f in range(4)) + "};\n")
        out.append(f"static __constant__ double kFacetLoadW{P}[4][4][{nd}] = {{" +
                   ", ".join("{" + ", ".join("{" + ", ".join(lit(x) for x in row) + "}" for row in wl[f]) + "}"
                             for f in range(4)) + "};\n")
    out.append("#endif  // FE_FACET_TABLES\n\n")
    return "".join(out)


def gen() -> str:
    out = []
    w = out.append
    w("// GENERATED by gen_element_code.py -- do not edit.\n")
    w("#pragma once\n\n")
    w("namespace fe {\n\n")
    # integrals of the P2 basis
    ints = [pint(p) for p in PHI]
    w("// int_ref phi_i (reference volume 1/6)\n")
    w("__device__ __forceinline__ double p2_basis_integral(int i) {\n")
    w("  return i < 4 ? " + lit(ints[0]) + " : " + lit(ints[4]) + ";\n}\n\n")

    # P3: basis integrals and stiffness with a cellwise-constant coefficient
    ints3 = [pint(p) for p in PHI3]
    w("// int_ref phi_i of the equispaced P3 element (vertices, edge pairs, faces)\n")
    w("__device__ __forceinline__ double p3_basis_integral(int i) {\n")
    w("  return i < 4 ? " + lit(ints3[0]) + " : (i < 16 ? " + lit(ints3[4]) + " : " + lit(ints3[16]) + ");\n}\n\n")
    w("// P3 stiffness with a cellwise-constant coefficient: g[s] = k * Ghat_s;\n")
    w("// emit(i, j, value) for the 210 unique entries i <= j.\n")
    w("template <typename T, typename Emit>\n")
    w("__device__ __forceinline__ void p3_stiffness_const(const T* g, Emit&& emit) {\n")
    exprs3 = {}
    maxabs3 = Fraction(0)
    for (i, j) in UNIQ3:
        terms = []
        for s_ in range(6):
            c = sym_pair(r3_plain, s_, i, j)
            if c != 0:
                terms.append((s_, c))
                maxabs3 = max(maxabs3, abs(c))
        exprs3[(i, j)] = sum_expr('g', terms, 2)
    w(symmetric_body(exprs3, 20))
    w("}\n")
    w(f"constexpr double kP3ConstTermMax = {lit(maxabs3)};\n\n")
    # the same coefficients as a table for kernels that evaluate entries lane
    # by lane: kP3GradGradSym[s*400 + i*20 + j] (every (i, j), so the table
    # is symmetric in i, j entry for entry)
    w("// P3 stiffness coefficients by geometry pair s: entry (i, j) = sum_s g[s] *\n")
    w("// kP3GradGradSym[s*400 + i*20 + j] (the terms of p3_stiffness_const).\n")
    w("__device__ const double kP3GradGradSym[2400] = {\n")
    vals3 = [lit(sym_pair(r3_plain, s_, i, j)) for s_ in range(6) for i in range(20) for j in range(20)]
    for k in range(0, 2400, 6):
        w("    " + ", ".join(vals3[k:k + 6]) + ",\n")
    w("};\n\n")

    # P2 stiffness, P1 coefficient: q[m*6+s] = k_m * Ghat_s
    w("// P2 stiffness with a P1 coefficient: q[m*6+s] = k_m * Ghat_s,\n")
    w("// Ghat = |detJ| K K^T (s over (00,11,22,01,02,12)).  Calls emit(i, j, value)\n")
    w("// for the 55 unique entries i <= j (FP32: off-diagonal entries first, then\n")
    w("// the diagonal entries as minus their rows' FP64 sums; emit takes a double).\n")
    w("template <typename T, typename Emit>\n")
    w("__device__ __forceinline__ void p2_stiffness_p1coef(const T* q, Emit&& emit) {\n")
    nterms = 0
    maxabs_p1coef = Fraction(0)
    exprs = {}
    for (i, j) in UNIQ:
        terms = []
        for m in range(4):
            for s in range(6):
                c = sym_pair(lambda a, b, ii, jj: r_weighted(m, a, b, ii, jj), s, i, j)
                if c != 0:
                    terms.append((m * 6 + s, c))
                    maxabs_p1coef = max(maxabs_p1coef, abs(c))
        nterms += len(terms)
        exprs[(i, j)] = sum_expr('q', terms)
    w(symmetric_body(exprs, 10))
    w("}\n")
    w(f"// terms: {nterms}\n\n")

    # P2 stiffness, cellwise-constant coefficient: g[s] = k * Ghat_s
    w("// P2 stiffness with a cellwise-constant coefficient: g[s] = k * Ghat_s.\n")
    w("template <typename T, typename Emit>\n")
    w("__device__ __forceinline__ void p2_stiffness_const(const T* g, Emit&& emit) {\n")
    maxabs_const = Fraction(0)
    exprs = {}
    for (i, j) in UNIQ:
        terms = []
        for s in range(6):
            c = sym_pair(r_plain, s, i, j)
            if c != 0:
                terms.append((s, c))
                maxabs_const = max(maxabs_const, abs(c))
        exprs[(i, j)] = sum_expr('g', terms, 2)
    w(symmetric_body(exprs, 10))
    w("}\n\n")
    w("// Largest |coefficient| of the two P2 stiffness bodies: |A_ij| <= max * sum|q| bounds every entry.\n")
    w(f"constexpr double kP2P1CoefTermMax = {lit(maxabs_p1coef)};\n")
    w(f"constexpr double kP2ConstTermMax = {lit(maxabs_const)};\n\n")

    # vector P2 elasticity: block (a,b), entry (i,j): sum_pq W[p*3+q] R0[p][q][i][j]
    w("// One 10x10 block of vector-P2 elasticity: value(i,j) = sum_pq W[p*3+q] *\n")
    w("// int_ref d_p phi_i d_q phi_j.  full=false emits only i <= j (diagonal blocks).\n")
    for full in (True, False):
        name = "p2_block_full" if full else "p2_block_upper"
        w("template <typename T, typename Emit>\n")
        w(f"__device__ __forceinline__ void {name}(const T* W, Emit&& emit) {{\n")
        exprs = {}
        for i in range(10):
            for j in range(10) if full else range(i, 10):
                terms = []
                for p in range(3):
                    for q in range(3):
                        c = r_plain(p, q, i, j)
                        if c != 0:
                            terms.append((p * 3 + q, c))
                exprs[(i, j)] = sum_expr('W', terms, 2)
        w(full_body(exprs, 10) if full else symmetric_body(exprs, 10))
        w("}\n\n")
    # the same reference integrals as a table, for kernels that evaluate block
    # entries lane by lane: kP2GradGrad[(i*10 + j)*9 + p*3 + q] = int_ref d_p phi_i d_q phi_j
    w("// int_ref d_p phi_i d_q phi_j of the P2 basis, index (i*10 + j)*9 + p*3 + q.\n")
    w("__device__ const double kP2GradGrad[900] = {\n")
    vals = [lit(r_plain(p_, q_, i, j)) for i in range(10) for j in range(10) for p_ in range(3) for q_ in range(3)]
    for k in range(0, 900, 6):
        w("    " + ", ".join(vals[k:k + 6]) + ",\n")
    w("};\n\n")
    w(mass_tables())
    w(facet_tables())
    w("}  // namespace fe\n")
    return "".join(out)


def plain_symmetric_body(exprs):
    """Body emitting the unique entries i <= j from their expressions in
    every precision (mass blocks have no zero row sums to preserve)."""
    return "".join(f"  emit({i}, {j}, {e});\n" for (i, j), e in exprs.items())


def mass_tables() -> str:
    """Mass matrices c*u*v*dx of P1 and P2 with a cellwise-constant or a P1
    coefficient, from the exact reference integrals (reference volume 1/6):
    const: s = c |det J|, entry = s int_ref phi_i phi_j;
    P1:    cq[m] = c_m |det J|, entry = sum_m cq[m] int_ref lambda_m phi_i phi_j."""
    out = []
    w = out.append
    for name, basis in (("p1", LAM), ("p2", PHI)):
        n = len(basis)
        uniq = [(i, j) for i in range(n) for j in range(i, n)]
        w(f"// {name.upper()} mass, cellwise-constant coefficient: s = c * |det J|; emit(i, j, value), i <= j.\n")
        w("template <typename T, typename Emit>\n")
        w(f"__device__ __forceinline__ void {name}_mass_const(T s, Emit&& emit) {{\n")
        exprs = {}
        for (i, j) in uniq:
            c = pint(pmul(basis[i], basis[j]))
            exprs[(i, j)] = f"s * T({lit(c)})" if c != 0 else "T(0)"
        w(plain_symmetric_body(exprs))
        w("}\n")
        w(f"// {name.upper()} mass, P1 coefficient: cq[m] = c_m * |det J|.\n")
        w("template <typename T, typename Emit>\n")
        w(f"__device__ __forceinline__ void {name}_mass_p1coef(const T* cq, Emit&& emit) {{\n")
        exprs = {}
        for (i, j) in uniq:
            terms = []
            for m in range(4):
                c = pint(pmul(LAM[m], pmul(basis[i], basis[j])))
                if c != 0:
                    terms.append((m, c))
            exprs[(i, j)] = sum_expr("cq", terms, 2)
        w(plain_symmetric_body(exprs))
        w("}\n\n")
    return "".join(out)


def main(argv):
    here = os.path.dirname(os.path.abspath(__file__))
    dst = argv[1] if len(argv) > 1 else os.path.join(here, "fe_element_code.cuh")
    text = gen()
    if not os.path.exists(dst) or open(dst).read() != text:
        with open(dst, "w") as fh:
            fh.write(text)


if __name__ == "__main__":
    main(sys.argv)
