"""Hand-written tabulate_tensor bodies in FFCx's format, for the tests of forms
given as FFCx bodies (fe_form_create_ffcx).

FFCx is not installed here, so these bodies stand in for what it generates
from UFL: the body of a ``tabulate_tensor_integral_*`` function with FFCx's
signature (A, w, c, coordinate_dofs, entity_local_index,
quadrature_permutation), static const tables of basis values and reference
derivatives laid out [permutation][entity][point][dof] as FFCx lays them out,
the Jacobian from the P1 coordinate element, and ``A[...] +=`` accumulation
(the caller zeroes A).  Element layouts follow FFCx / DOLFINx: blocked
elements interleave components (dof*bs + comp), interior facets use macro
dofs (cell 0's then cell 1's) and macro coefficients (per coefficient cell
0's values then cell 1's), and coordinate_dofs holds 4 vertices x 3
coordinates per cell.  Quadrature rules and tables come from the oracle
(fem_oracle.tet_rule / tri_rule / lagrange_tables), whose independent numpy
evaluation of the same forms is the reference the engine is checked against.

Each builder returns dict(name, body, integral_type, rank, coefficient_sizes,
num_constants).
"""
from __future__ import annotations

import hashlib

import numpy as np

from oracle import fem_oracle as fo

CELL, EXTERIOR, INTERIOR = "cell", "exterior_facet", "interior_facet"


def _fmt(v):
    return repr(float(v))


def _array(name, a):
    a = np.asarray(a, dtype=float)
    dims = "".join(f"[{d}]" for d in a.shape)

    def rec(x):
        if x.ndim == 1:
            return "{" + ", ".join(_fmt(v) for v in x) + "}"
        return "{" + ", ".join(rec(y) for y in x) + "}"

    return f"alignas(16) static const double {name}{dims} = {rec(a)};\n"


def _name(tag, body):
    return "tabulate_tensor_integral_" + tag + "_" + hashlib.sha1(body.encode()).hexdigest()[:10]


def _geometry(off=0, suffix=""):
    """Jacobian J, |det J| and K = J^-1 of the cell whose coordinates start at
    coordinate_dofs[off] (P1 coordinate element: constant derivatives)."""
    s = suffix
    return f"""  // Jacobian of the affine map (coordinate element derivatives FE_CG_D)
  double J{s}[3][3];
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) {{
      double acc = 0.0;
      for (int v = 0; v < 4; ++v) acc += coordinate_dofs[{off} + 3 * v + r] * FE_CG_D[v][k];
      J{s}[r][k] = acc;
    }}
  const double detJ{s} = J{s}[0][0] * (J{s}[1][1] * J{s}[2][2] - J{s}[1][2] * J{s}[2][1])
                     - J{s}[0][1] * (J{s}[1][0] * J{s}[2][2] - J{s}[1][2] * J{s}[2][0])
                     + J{s}[0][2] * (J{s}[1][0] * J{s}[2][1] - J{s}[1][1] * J{s}[2][0]);
  double K{s}[3][3];
  K{s}[0][0] = (J{s}[1][1] * J{s}[2][2] - J{s}[1][2] * J{s}[2][1]) / detJ{s};
  K{s}[0][1] = (J{s}[0][2] * J{s}[2][1] - J{s}[0][1] * J{s}[2][2]) / detJ{s};
  K{s}[0][2] = (J{s}[0][1] * J{s}[1][2] - J{s}[0][2] * J{s}[1][1]) / detJ{s};
  K{s}[1][0] = (J{s}[1][2] * J{s}[2][0] - J{s}[1][0] * J{s}[2][2]) / detJ{s};
  K{s}[1][1] = (J{s}[0][0] * J{s}[2][2] - J{s}[0][2] * J{s}[2][0]) / detJ{s};
  K{s}[1][2] = (J{s}[0][2] * J{s}[1][0] - J{s}[0][0] * J{s}[1][2]) / detJ{s};
  K{s}[2][0] = (J{s}[1][0] * J{s}[2][1] - J{s}[1][1] * J{s}[2][0]) / detJ{s};
  K{s}[2][1] = (J{s}[0][1] * J{s}[2][0] - J{s}[0][0] * J{s}[2][1]) / detJ{s};
  K{s}[2][2] = (J{s}[0][0] * J{s}[1][1] - J{s}[0][1] * J{s}[1][0]) / detJ{s};
"""


_CG_D = _array("FE_CG_D", [[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


def _cell_tables(degree, tag, X):
    V, D = fo.lagrange_tables(degree, X)
    return (_array(f"FE{tag}_V", V[None, None]) +  # [1][1][N][k]
            _array(f"FE{tag}_D", np.transpose(D, (2, 0, 1))[None, None]))  # [1][1][3][N][k]


def _facet_tables(degree, tag, P2, perms):
    """Tables [perm][facet][N][k] (values) and [perm][facet][3][N][k] (reference
    derivatives) at the rule's points on each local facet, for each quadrature
    permutation (perms = 1: no permutation)."""
    Vs, Ds = [], []
    for p in range(perms):
        Pp = fo.permute_facet_points(P2, p) if perms > 1 else P2
        vv, dd = [], []
        for f in range(4):
            V, D = fo.lagrange_tables(degree, fo.facet_points(f, Pp))
            vv.append(V)
            dd.append(np.transpose(D, (2, 0, 1)))
        Vs.append(vv)
        Ds.append(dd)
    return _array(f"FE{tag}_V", np.array(Vs)) + _array(f"FE{tag}_D", np.array(Ds))


def _grad(tag, n, dst, K="K", p="0", f="0", q="iq"):
    """dst[i][a] = sum_b K[b][a] * FE_D[p][f][b][q][i]: physical gradients of n basis functions."""
    return (f"    double {dst}[{n}][3];\n"
            f"    for (int i = 0; i < {n}; ++i)\n"
            f"      for (int a = 0; a < 3; ++a)\n"
            f"        {dst}[i][a] = {K}[0][a] * FE{tag}_D[{p}][{f}][0][{q}][i] + {K}[1][a] * FE{tag}_D[{p}][{f}][1][{q}][i]"
            f" + {K}[2][a] * FE{tag}_D[{p}][{f}][2][{q}][i];\n")


def _build(tag, itype, rank, sizes, nconst, body):
    return dict(name=_name(tag, body), body=body, integral_type=itype, rank=rank, coefficient_sizes=list(sizes),
                num_constants=nconst)


# ---------------------------------------------------------------------------
# cell integrals
# ---------------------------------------------------------------------------
def stiffness(degree: int, k_kind: str = "dg0", qdeg: int = 3):
    """k * inner(grad u, grad v) * dx on scalar Lagrange `degree`; k a DG0 field
    (w[0]) or a P1 field (w[0..3])."""
    X, w = fo.tet_rule(qdeg)
    kd = 4 if k_kind == "p1" else 1
    nd = {1: 4, 2: 10, 3: 20}[degree]
    body = ("  // Quadrature rules\n" + _array("weights_c", w) +
            "  // Precomputed values of basis functions\n" + _CG_D + _cell_tables(degree, "U", X) +
            (_cell_tables(1, "K", X) if k_kind == "p1" else "") +
            _geometry() +
            f"  for (int iq = 0; iq < {len(w)}; ++iq) {{\n" +
            ("    double k = 0.0;\n    for (int m = 0; m < 4; ++m) k += w[m] * FEK_V[0][0][iq][m];\n"
             if k_kind == "p1" else "    const double k = w[0];\n") +
            _grad("U", nd, "G") +
            "    const double fw = k * fabs(detJ) * weights_c[iq];\n"
            f"    for (int i = 0; i < {nd}; ++i)\n"
            f"      for (int j = 0; j < {nd}; ++j)\n"
            f"        A[i * {nd} + j] += fw * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]);\n"
            "  }\n")
    return _build(f"stiff{degree}{k_kind}", CELL, 2, [kd], 0, body)


def stiffness_plus_mass():
    """k * inner(grad u, grad v) * dx + c * u * v * dx on P1, k DG0 (w[0]),
    c a Constant (c[0]): a form none of the built-in kinds has."""
    X, w = fo.tet_rule(3)
    body = ("  // Quadrature rules\n" + _array("weights_c", w) + _CG_D + _cell_tables(1, "U", X) + _geometry() +
            f"  for (int iq = 0; iq < {len(w)}; ++iq) {{\n" + _grad("U", 4, "G") +
            "    const double dx = fabs(detJ) * weights_c[iq];\n"
            "    for (int i = 0; i < 4; ++i)\n"
            "      for (int j = 0; j < 4; ++j)\n"
            "        A[i * 4 + j] += dx * (w[0] * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2])\n"
            "                              + c[0] * FEU_V[0][0][iq][i] * FEU_V[0][0][iq][j]);\n"
            "  }\n")
    return _build("stiffmass", CELL, 2, [1], 1, body)


def elasticity():
    """2 mu eps(u):eps(v) + lam div(u) div(v) on vector P2 (blocked, bs 3),
    lam = w[0], mu = w[1] (DG0)."""
    X, w = fo.tet_rule(3)
    body = ("  // Quadrature rules\n" + _array("weights_c", w) + _CG_D + _cell_tables(2, "U", X) + _geometry() +
            f"  for (int iq = 0; iq < {len(w)}; ++iq) {{\n" + _grad("U", 10, "G") +
            "    const double dx = fabs(detJ) * weights_c[iq];\n"
            "    const double lam = w[0], mu = w[1];\n"
            "    for (int i = 0; i < 10; ++i)\n"
            "      for (int a = 0; a < 3; ++a)\n"
            "        for (int j = 0; j < 10; ++j)\n"
            "          for (int b = 0; b < 3; ++b) {\n"
            "            // eps(phi_j e_b) : eps(phi_i e_a) and div terms\n"
            "            double gg = G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2];\n"
            "            double v = mu * ((a == b ? gg : 0.0) + G[i][b] * G[j][a]) + lam * G[i][a] * G[j][b];\n"
            "            A[(3 * i + a) * 30 + 3 * j + b] += dx * v;\n"
            "          }\n"
            "  }\n")
    return _build("elast", CELL, 2, [1, 1], 0, body)


def mixed_p2_p1():
    """int p * d(v)/dx dx: test v in P2, trial p in P1 (a 10 x 4 coupling block
    of a mixed system)."""
    X, w = fo.tet_rule(3)
    body = ("  // Quadrature rules\n" + _array("weights_c", w) + _CG_D + _cell_tables(2, "V", X) +
            _cell_tables(1, "P", X) + _geometry() +
            f"  for (int iq = 0; iq < {len(w)}; ++iq) {{\n" + _grad("V", 10, "G") +
            "    const double dx = fabs(detJ) * weights_c[iq];\n"
            "    for (int i = 0; i < 10; ++i)\n"
            "      for (int j = 0; j < 4; ++j) A[i * 4 + j] += dx * G[i][0] * FEP_V[0][0][iq][j];\n"
            "  }\n")
    return _build("mixed21", CELL, 2, [], 0, body)


def _nl_point():
    """u, grad u, kappa at the point from the packed coefficients w = (u, kappa), both P1."""
    return ("    double u = 0.0, kap = 0.0, gu[3] = {0.0, 0.0, 0.0};\n"
            "    for (int m = 0; m < 4; ++m) {\n"
            "      u += w[m] * FEU_V[0][0][iq][m];\n"
            "      kap += w[4 + m] * FEU_V[0][0][iq][m];\n"
            "      for (int a = 0; a < 3; ++a) gu[a] += w[m] * G[m][a];\n"
            "    }\n")


def nonlinear(rank: int, n: int = 4):
    """The reference's cell test forms (python/test/test_cuda_assembly.py:48-91)
    on P1 tetrahedra, u and kappa P1 coefficients (w = u, kappa):
    rank 1: (exp(u) kappa v + grad u . grad v) dx;  rank 2: its derivative in u;
    rank 0: exp(u) kappa dx."""
    X, w = fo.tet_rule(n)
    head = "  // Quadrature rules\n" + _array("weights_c", w) + _CG_D + _cell_tables(1, "U", X) + _geometry()
    loop = f"  for (int iq = 0; iq < {len(w)}; ++iq) {{\n" + _grad("U", 4, "G") + _nl_point()
    loop += "    const double dx = fabs(detJ) * weights_c[iq];\n    const double e = exp(u) * kap * dx;\n"
    if rank == 0:
        loop += "    A[0] += e;\n"
    elif rank == 1:
        loop += ("    for (int i = 0; i < 4; ++i)\n"
                 "      A[i] += e * FEU_V[0][0][iq][i] + dx * (gu[0] * G[i][0] + gu[1] * G[i][1] + gu[2] * G[i][2]);\n")
    else:
        loop += ("    for (int i = 0; i < 4; ++i)\n"
                 "      for (int j = 0; j < 4; ++j)\n"
                 "        A[i * 4 + j] += e * FEU_V[0][0][iq][j] * FEU_V[0][0][iq][i]\n"
                 "                        + dx * (G[j][0] * G[i][0] + G[j][1] * G[i][1] + G[j][2] * G[i][2]);\n")
    return _build(f"nl{rank}", CELL, rank, [4, 4], 0, head + loop + "  }\n")


# ---------------------------------------------------------------------------
# facet integrals
# ---------------------------------------------------------------------------
def _facet_normal(off=0, suffix="", f="entity_local_index[0]"):
    """Outward unit normal n and |J_F| (twice the facet area) of local facet f
    of the cell at coordinate_dofs[off]."""
    s = suffix
    return f"""    // facet f = {{0,1,2,3}} minus f, vertices in increasing local order; the
    // normal points away from the vertex off the facet
    static const int facet_vertices[4][3] = {{{{1, 2, 3}}, {{0, 2, 3}}, {{0, 1, 3}}, {{0, 1, 2}}}};
    const int lf{s} = {f};
    const double* p0{s} = coordinate_dofs + {off} + 3 * facet_vertices[lf{s}][0];
    const double* p1{s} = coordinate_dofs + {off} + 3 * facet_vertices[lf{s}][1];
    const double* p2{s} = coordinate_dofs + {off} + 3 * facet_vertices[lf{s}][2];
    const double* po{s} = coordinate_dofs + {off} + 3 * lf{s};
    double e1{s}[3], e2{s}[3], n{s}[3];
    for (int a = 0; a < 3; ++a) {{ e1{s}[a] = p1{s}[a] - p0{s}[a]; e2{s}[a] = p2{s}[a] - p0{s}[a]; }}
    n{s}[0] = e1{s}[1] * e2{s}[2] - e1{s}[2] * e2{s}[1];
    n{s}[1] = e1{s}[2] * e2{s}[0] - e1{s}[0] * e2{s}[2];
    n{s}[2] = e1{s}[0] * e2{s}[1] - e1{s}[1] * e2{s}[0];
    const double detJF{s} = sqrt(n{s}[0] * n{s}[0] + n{s}[1] * n{s}[1] + n{s}[2] * n{s}[2]);
    const double side{s} = (n{s}[0] * (p0{s}[0] - po{s}[0]) + n{s}[1] * (p0{s}[1] - po{s}[1]) + n{s}[2] * (p0{s}[2] - po{s}[2])) > 0.0 ? 1.0 : -1.0;
    for (int a = 0; a < 3; ++a) n{s}[a] *= side{s} / detJF{s};
"""


def robin_mass(degree: int = 1):
    """alpha * u * v * ds on scalar Lagrange `degree`, alpha a DG0 field (w[0])."""
    P2, w = fo.tri_rule(3)
    nd = {1: 4, 2: 10}[degree]
    body = ("  // Quadrature rules\n" + _array("weights_f", w) + _facet_tables(degree, "U", P2, 1) +
            f"  {{\n" + _facet_normal() +
            f"    for (int iq = 0; iq < {len(w)}; ++iq) {{\n"
            "      const double ds = w[0] * detJF * weights_f[iq];\n"
            f"      for (int i = 0; i < {nd}; ++i)\n"
            f"        for (int j = 0; j < {nd}; ++j)\n"
            f"          A[i * {nd} + j] += ds * FEU_V[0][lf][iq][i] * FEU_V[0][lf][iq][j];\n"
            "    }\n  }\n")
    return _build(f"robin{degree}", EXTERIOR, 2, [1], 0, body)


def exterior_nonlinear(rank: int):
    """The reference's exterior-facet test form u kappa v (grad u . n) ds and its
    derivative in u, on P1 (w = u, kappa)."""
    P2, w = fo.tri_rule(3)
    body = ("  // Quadrature rules\n" + _array("weights_f", w) + _CG_D + _facet_tables(1, "U", P2, 1) + _geometry() +
            "  {\n" + _facet_normal() +
            "    double G[4][3], gu[3] = {0.0, 0.0, 0.0}, gun = 0.0, gpn[4];\n"
            "    for (int i = 0; i < 4; ++i)\n"
            "      for (int a = 0; a < 3; ++a) G[i][a] = K[0][a] * FE_CG_D[i][0] + K[1][a] * FE_CG_D[i][1] + K[2][a] * FE_CG_D[i][2];\n"
            "    for (int m = 0; m < 4; ++m)\n      for (int a = 0; a < 3; ++a) gu[a] += w[m] * G[m][a];\n"
            "    for (int a = 0; a < 3; ++a) gun += gu[a] * n[a];\n"
            "    for (int j = 0; j < 4; ++j) gpn[j] = G[j][0] * n[0] + G[j][1] * n[1] + G[j][2] * n[2];\n"
            f"    for (int iq = 0; iq < {len(w)}; ++iq) {{\n"
            "      double u = 0.0, kap = 0.0;\n"
            "      for (int m = 0; m < 4; ++m) { u += w[m] * FEU_V[0][lf][iq][m]; kap += w[4 + m] * FEU_V[0][lf][iq][m]; }\n"
            "      const double ds = detJF * weights_f[iq];\n")
    if rank == 1:
        body += "      for (int i = 0; i < 4; ++i) A[i] += ds * u * kap * FEU_V[0][lf][iq][i] * gun;\n"
    else:
        body += ("      for (int i = 0; i < 4; ++i)\n"
                 "        for (int j = 0; j < 4; ++j)\n"
                 "          A[i * 4 + j] += ds * kap * FEU_V[0][lf][iq][i] * (FEU_V[0][lf][iq][j] * gun + u * gpn[j]);\n")
    body += "    }\n  }\n"
    return _build(f"extnl{rank}", EXTERIOR, rank, [4, 4], 0, body)


def _interior_head(degree_tag_pairs):
    P2, w = fo.tri_rule(3)
    head = "  // Quadrature rules\n" + _array("weights_f", w) + _CG_D
    for deg, tag in degree_tag_pairs:
        head += _facet_tables(deg, tag, P2, 6)
    return head, len(w)


def interior_jump():
    """alpha * jump(u) * jump(v) * dS on DG1 (jump = cell 0 minus cell 1);
    alpha a Constant (c[0])."""
    head, nq = _interior_head([(1, "U")])
    body = (head + "  {\n" + _facet_normal() +
            "    const int lf1 = entity_local_index[1];\n"
            "    const int qp0 = quadrature_permutation[0], qp1 = quadrature_permutation[1];\n"
            f"    for (int iq = 0; iq < {nq}; ++iq) {{\n"
            "      const double ds = c[0] * detJF * weights_f[iq];\n"
            "      double jmp[8];\n"
            "      for (int i = 0; i < 4; ++i) { jmp[i] = FEU_V[qp0][lf][iq][i]; jmp[4 + i] = -FEU_V[qp1][lf1][iq][i]; }\n"
            "      for (int i = 0; i < 8; ++i)\n"
            "        for (int j = 0; j < 8; ++j) A[i * 8 + j] += ds * jmp[i] * jmp[j];\n"
            "    }\n  }\n")
    return _build("ijump", INTERIOR, 2, [], 1, body)


def interior_sipg():
    """-avg(grad u . n) jump(v) - jump(u) avg(grad v . n) + alpha jump(u) jump(v)
    on DG1 (n out of cell 0), alpha a Constant (c[0])."""
    head, nq = _interior_head([(1, "U")])
    body = (head + _geometry(0, "0") + _geometry(12, "1") + "  {\n" + _facet_normal() +
            "    const int lf1 = entity_local_index[1];\n"
            "    const int qp0 = quadrature_permutation[0], qp1 = quadrature_permutation[1];\n"
            "    double agn[8];  // avg(grad phi . n) of the macro basis\n"
            "    for (int i = 0; i < 4; ++i) {\n"
            "      double g0 = 0.0, g1 = 0.0;\n"
            "      for (int a = 0; a < 3; ++a) {\n"
            "        g0 += (K0[0][a] * FE_CG_D[i][0] + K0[1][a] * FE_CG_D[i][1] + K0[2][a] * FE_CG_D[i][2]) * n[a];\n"
            "        g1 += (K1[0][a] * FE_CG_D[i][0] + K1[1][a] * FE_CG_D[i][1] + K1[2][a] * FE_CG_D[i][2]) * n[a];\n"
            "      }\n"
            "      agn[i] = 0.5 * g0;\n      agn[4 + i] = 0.5 * g1;\n"
            "    }\n"
            f"    for (int iq = 0; iq < {nq}; ++iq) {{\n"
            "      const double ds = detJF * weights_f[iq];\n"
            "      double jmp[8];\n"
            "      for (int i = 0; i < 4; ++i) { jmp[i] = FEU_V[qp0][lf][iq][i]; jmp[4 + i] = -FEU_V[qp1][lf1][iq][i]; }\n"
            "      for (int i = 0; i < 8; ++i)\n"
            "        for (int j = 0; j < 8; ++j)\n"
            "          A[i * 8 + j] += ds * (-agn[j] * jmp[i] - jmp[j] * agn[i] + c[0] * jmp[i] * jmp[j]);\n"
            "    }\n  }\n")
    return _build("sipg", INTERIOR, 2, [], 1, body)


def interior_nonlinear(rank: int):
    """The reference's interior-facet test forms on DG1 with a P1 kappa,
    w = (u [DG1], kappa [P1]) in macro layout (u cell 0, u cell 1, kappa cell 0,
    kappa cell 1): rank 0: avg(u^2) avg(kappa) dS; rank 1: avg(v) avg(kappa)
    avg(u^2) dS; rank 2: its derivative in u."""
    head, nq = _interior_head([(1, "U")])
    body = (head + "  {\n" + _facet_normal() +
            "    const int lf1 = entity_local_index[1];\n"
            "    const int qp0 = quadrature_permutation[0], qp1 = quadrature_permutation[1];\n"
            f"    for (int iq = 0; iq < {nq}; ++iq) {{\n"
            "      double u0 = 0.0, u1 = 0.0, k0 = 0.0, k1 = 0.0;\n"
            "      for (int m = 0; m < 4; ++m) {\n"
            "        u0 += w[m] * FEU_V[qp0][lf][iq][m];\n        u1 += w[4 + m] * FEU_V[qp1][lf1][iq][m];\n"
            "        k0 += w[8 + m] * FEU_V[qp0][lf][iq][m];\n        k1 += w[12 + m] * FEU_V[qp1][lf1][iq][m];\n"
            "      }\n"
            "      const double ds = detJF * weights_f[iq];\n"
            "      const double kav = 0.5 * (k0 + k1), u2av = 0.5 * (u0 * u0 + u1 * u1);\n")
    if rank == 0:
        body += "      A[0] += ds * u2av * kav;\n"
    else:
        body += ("      double av[8];\n"
                 "      for (int i = 0; i < 4; ++i) { av[i] = 0.5 * FEU_V[qp0][lf][iq][i]; av[4 + i] = 0.5 * FEU_V[qp1][lf1][iq][i]; }\n")
        if rank == 1:
            body += "      for (int i = 0; i < 8; ++i) A[i] += ds * av[i] * kav * u2av;\n"
        else:
            body += ("      double du[8];\n"
                     "      for (int j = 0; j < 4; ++j) { du[j] = u0 * FEU_V[qp0][lf][iq][j]; du[4 + j] = u1 * FEU_V[qp1][lf1][iq][j]; }\n"
                     "      for (int i = 0; i < 8; ++i)\n"
                     "        for (int j = 0; j < 8; ++j) A[i * 8 + j] += ds * av[i] * kav * du[j];\n")
    body += "    }\n  }\n"
    return _build(f"inl{rank}", INTERIOR, rank, [4, 4], 0, body)
