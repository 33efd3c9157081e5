"""Generates lag2d_tables.inc: exact constant tables of the 9-node quad.

The 9-node quad map is the tensor product of the 1-D quadratic Lagrange
polynomials L0(r) = r(r-1)/2, L1(r) = 1-r^2, L2(r) = r(r+1)/2 (node k of the
reference ordering sits at the tensor index NODE_AB[k]).  Its Jacobian
determinant is the bilinear form

    det J(r,s) = sum_{i<j} (x_i y_j - x_j y_i) A_ij(r,s),
    A_ij = dNi/dr dNj/ds - dNi/ds dNj/dr,

a polynomial of degree <= 3 in r and in s.  The tables give, with rational
arithmetic rounded once to double:

  detpoly    the 16 coefficients of det J as a fixed linear map of the 36
             node cross products (coefficient of r^m s^n of A_{i<j});
  subareas   the exact area of each sub-cell (the 9-node sub-quad the
             reference builds in getrhosubg_averg, Getrhslaggauss.f90:
             7185-7257) as a linear form of the parent cross products;
  cell_area  the exact area of the cell from the det J coefficients.
emitted as straight-line code (zero coefficients dropped).

Run:  python lag2d_b200/csrc/gen_tables.py   (writes lag2d_tables.inc here)
"""
from fractions import Fraction as F
import itertools
import os

HERE = os.path.dirname(os.path.abspath(__file__))

# reference node k -> (a, b): r index a, s index b in {0: -1, 1: 0, 2: +1}
NODE_AB = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]

# 1-D Lagrange polynomials as coefficient lists (ascending powers)
L = [[F(0), F(-1, 2), F(1, 2)], [F(1), F(0), F(-1)], [F(0), F(1, 2), F(1, 2)]]


def pmul(a, b):
    out = [F(0)] * (len(a) + len(b) - 1)
    for i, x in enumerate(a):
        for j, y in enumerate(b):
            out[i + j] += x * y
    return out


def pder(a):
    return [i * a[i] for i in range(1, len(a))] or [F(0)]


def peval(a, x):
    return sum(c * x ** i for i, c in enumerate(a))


def shape2(k):
    """N_k as dict {(m, n): coeff} of r^m s^n."""
    a, b = NODE_AB[k]
    return {(m, n): L[a][m] * L[b][n] for m in range(3) for n in range(3) if L[a][m] * L[b][n] != 0}


def d_r(p):
    return {(m - 1, n): m * c for (m, n), c in p.items() if m > 0}


def d_s(p):
    return {(m, n - 1): n * c for (m, n), c in p.items() if n > 0}


def mul2(p, q):
    out = {}
    for (m1, n1), c1 in p.items():
        for (m2, n2), c2 in q.items():
            out[(m1 + m2, n1 + n2)] = out.get((m1 + m2, n1 + n2), F(0)) + c1 * c2
    return out


def sub2(p, q):
    out = dict(p)
    for k, c in q.items():
        out[k] = out.get(k, F(0)) - c
    return {k: c for k, c in out.items() if c != 0}


PAIRS = [(i, j) for i in range(9) for j in range(i + 1, 9)]


def detp_table():
    N = [shape2(k) for k in range(9)]
    tab = []
    for i, j in PAIRS:
        A = sub2(mul2(d_r(N[i]), d_s(N[j])), mul2(d_s(N[i]), d_r(N[j])))
        row = [A.get((m, n), F(0)) for m in range(4) for n in range(4)]
        tab.append(row)
    return tab


def integ(poly, r0, r1, s0, s1):
    """Exact integral of {(m,n): c} over [r0,r1] x [s0,s1]."""
    tot = F(0)
    for (m, n), c in poly.items():
        tot += c * (F(r1) ** (m + 1) - F(r0) ** (m + 1)) / (m + 1) * (F(s1) ** (n + 1) - F(s0) ** (n + 1)) / (n + 1)
    return tot


def sub_matrix(isg):
    """Sub-cell node k (reference order) as a linear combination of parent nodes (9 x 9)."""
    ipqsg = [[1, 5, 9, 8], [5, 2, 6, 9], [9, 6, 3, 7], [8, 9, 7, 4]][isg]
    posqc = [(-0.5, -1), (0.5, -1), (1, -0.5), (1, 0.5), (0.5, 1), (-0.5, 1), (-1, 0.5), (-1, -0.5),
             (0, -0.5), (0.5, 0), (0, 0.5), (-0.5, 0)]
    ipqsc = [[1, 9, 12, 8], [2, 3, 10, 9], [10, 4, 5, 11], [12, 11, 6, 7]][isg]
    N = [shape2(k) for k in range(9)]
    S = [[F(0)] * 9 for _ in range(9)]
    for k in range(4):
        S[k][ipqsg[k] - 1] = F(1)
        r, s = posqc[ipqsc[k] - 1]
        for p in range(9):
            S[4 + k][p] = sum(c * F(r) ** m * F(s) ** n for (m, n), c in N[p].items())
    for p in range(9):
        S[8][p] = F(-1, 4) * (S[0][p] + S[1][p] + S[2][p] + S[3][p]) + F(1, 2) * (S[4][p] + S[5][p] + S[6][p] + S[7][p])
    return S


def ksub_table():
    N = [shape2(k) for k in range(9)]
    # area of a 9-node quad with nodes (X, Y): sum_{a<b} (X_a Y_b - X_b Y_a) * Abar_ab
    Abar = {}
    for a, b in PAIRS:
        A = sub2(mul2(d_r(N[a]), d_s(N[b])), mul2(d_s(N[a]), d_r(N[b])))
        Abar[(a, b)] = integ(A, -1, 1, -1, 1)
    tab = []
    for isg in range(4):
        S = sub_matrix(isg)
        # X = S x, Y = S y: sum_{a<b} Abar_ab (X_a Y_b - X_b Y_a) = sum_{i,j} x_i y_j M_ij, M antisymmetric
        M = [[F(0)] * 9 for _ in range(9)]
        for (a, b), w in Abar.items():
            for i in range(9):
                for j in range(9):
                    M[i][j] += w * (S[a][i] * S[b][j] - S[b][i] * S[a][j])
        tab.append([M[i][j] for i, j in PAIRS])  # coefficient of (x_i y_j - x_j y_i)
    return tab


def cell_area_coeffs():
    """Area of the parent from the det J polynomial: sum_mn D_mn mu_m mu_n."""
    mu = [F(2), F(0), F(2, 3), F(0)]
    return [mu[m] * mu[n] for m in range(4) for n in range(4)]


def fmt(x):
    v = float(x)
    return repr(v) if v != int(v) else f"{int(v)}.0"


def lincomb(terms):
    """C++ expression sum of coeff * var, skipping zero coefficients."""
    parts = []
    for coef, var in terms:
        if coef == 0:
            continue
        if coef == 1:
            parts.append(var)
        elif coef == -1:
            parts.append(f"-{var}")
        else:
            parts.append(f"{fmt(coef)} * {var}")
    return " + ".join(parts).replace("+ -", "- ") if parts else "0.0"


def main():
    detp = detp_table()
    ksub = ksub_table()
    area = cell_area_coeffs()
    out = ["// Generated by gen_tables.py -- exact rationals rounded once to double.",
           "// c[p] = x_i y_j - x_j y_i for the node pair p = (PAIR_I[p], PAIR_J[p]), i < j.",
           "#pragma once"]
    pi = ", ".join(str(i) for i, _ in PAIRS)
    pj = ", ".join(str(j) for _, j in PAIRS)
    out.append("__host__ __device__ __forceinline__ void cross36(const double (*xp)[2], double *c) {")
    for p, (i, j) in enumerate(PAIRS):
        out.append(f"  c[{p}] = xp[{i}][0] * xp[{j}][1] - xp[{j}][0] * xp[{i}][1];")
    out.append("}")
    out.append("// coefficients D[m*4+n] of r^m s^n of det J")
    out.append("__host__ __device__ __forceinline__ void detpoly(const double *c, double *D) {")
    for t in range(16):
        out.append(f"  D[{t}] = {lincomb([(detp[p][t], f'c[{p}]') for p in range(36)])};")
    out.append("}")
    out.append("// exact area of sub-cell isg (the 9-node sub-quad of getrhosubg_averg)")
    out.append("__host__ __device__ __forceinline__ void subareas(const double *c, double *v) {")
    for isg in range(4):
        out.append(f"  v[{isg}] = {lincomb([(ksub[isg][p], f'c[{p}]') for p in range(36)])};")
    out.append("}")
    # transposed maps for the reverse (adjoint) pass: lc[p] += sum_t table[p][t] * l[t]
    out.append("// transpose of detpoly: lc[p] += sum_t dD[t]/dc[p] * lD[t]")
    out.append("__host__ __device__ __forceinline__ void detpoly_T(const double *lD, double *lc) {")
    for p in range(36):
        e = lincomb([(detp[p][t], f'lD[{t}]') for t in range(16)])
        if e != "0.0":
            out.append(f"  lc[{p}] += {e};")
    out.append("}")
    out.append("// transpose of subareas: lc[p] += sum_isg dv[isg]/dc[p] * lv[isg]")
    out.append("__host__ __device__ __forceinline__ void subareas_T(const double *lv, double *lc) {")
    for p in range(36):
        e = lincomb([(ksub[isg][p], f'lv[{isg}]') for isg in range(4)])
        if e != "0.0":
            out.append(f"  lc[{p}] += {e};")
    out.append("}")
    out.append("// exact area of the cell from det J coefficients")
    out.append("__host__ __device__ __forceinline__ double cell_area(const double *D) {")
    out.append(f"  return {lincomb([(area[t], f'D[{t}]') for t in range(16)])};")
    out.append("}")
    out.append(f"// pair order: i = {{{pi}}}, j = {{{pj}}}")
    with open(os.path.join(HERE, "lag2d_tables.inc"), "w") as f:
        f.write("\n".join(out) + "\n")
    nz = sum(1 for row in detp for v in row if v != 0)
    print(f"DETP nonzeros {nz} / {36 * 16}; KSUB nonzeros {sum(1 for r in ksub for v in r if v != 0)} / 144")


if __name__ == "__main__":
    main()
