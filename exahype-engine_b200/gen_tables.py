"""Generate csrc/exa_tables.cuh: the 1D Gauss-Legendre DG operators as device constants.

The operators are defined by the maths the reference's table generator uses
(Miscellaneous/aderdg/aderdg.py:14-195, generateLookupTable.py:146-182):

* nodes x_i and weights w_i of Gauss-Legendre quadrature on [0,1] (sum w = 1), ascending;
* Kxi[k][l] = sum_i w_i phi_k'(x_i) phi_l(x_i)          (stiffness, = w_l phi_k'(x_l));
* iK1 = (phi(1) phi(1)^T - Kxi)^{-1}                    (time-predictor solve, [row][col]);
* dudx = M^{-1} Kxi^T with M = diag(w)                  (nodal derivative);
* F0 = phi(0), F1 = phi(1)                              (extrapolation to the faces).

Evaluated here with mpmath at 50 digits and rounded to double, then written as one
``__constant__`` block per order. Run: ``python exahype-engine_b200/gen_tables.py``.
"""
import os

import mpmath as mp

mp.mp.dps = 50
MAX_ORDER = 9
HERE = os.path.dirname(os.path.abspath(__file__))


def gauss_legendre01(n):
    xs, ws = [], []
    for i in range(1, n + 1):
        # Newton on P_n from the Chebyshev-like initial guess
        x = mp.cos(mp.pi * (i - mp.mpf(1) / 4) / (n + mp.mpf(1) / 2))
        for _ in range(100):
            p0, p1 = mp.mpf(1), x
            for k in range(2, n + 1):
                p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
            dp = n * (x * p1 - p0) / (x * x - 1) if n > 1 else mp.mpf(1)
            dx = p1 / dp
            x -= dx
            if abs(dx) < mp.mpf(10) ** (-45):
                break
        p0, p1 = mp.mpf(1), x
        for k in range(2, n + 1):
            p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
        dp = n * (x * p1 - p0) / (x * x - 1) if n > 1 else mp.mpf(1)
        w = 2 / ((1 - x * x) * dp * dp) if n > 1 else mp.mpf(2)
        xs.append((1 - x) / 2)
        ws.append(w / 2)
    if n == 1:
        return [mp.mpf("0.5")], [mp.mpf(1)]
    return xs, ws


def basis(xin, xi):
    n = len(xin)
    phi = [mp.mpf(1)] * n
    dphi = [mp.mpf(0)] * n
    for m in range(n):
        for j in range(n):
            if j != m:
                phi[m] *= (xi - xin[j]) / (xin[m] - xin[j])
        for i in range(n):
            if i == m:
                continue
            t = mp.mpf(1)
            for j in range(n):
                if j in (i, m):
                    continue
                t *= (xi - xin[j]) / (xin[m] - xin[j])
            dphi[m] += t / (xin[m] - xin[i])
    return phi, dphi


def operators(order):
    n = order + 1
    x, w = gauss_legendre01(n)
    K = [[mp.mpf(0)] * n for _ in range(n)]
    for i in range(n):
        phi, dphi = basis(x, x[i])
        for k in range(n):
            for l in range(n):
                K[k][l] += w[i] * dphi[k] * phi[l]
    p1, _ = basis(x, mp.mpf(1))
    p0, _ = basis(x, mp.mpf(0))
    K1 = mp.matrix(n, n)
    for k in range(n):
        for l in range(n):
            K1[k, l] = p1[k] * p1[l] - K[k][l]
    iK1 = K1 ** -1
    dudx = [[K[j][i] / w[i] for j in range(n)] for i in range(n)]
    return dict(nodes=x, weights=w, Kxi=K, iK1=[[iK1[i, j] for j in range(n)] for i in range(n)], dudx=dudx,
                F0=p0, F1=p1)


def gauss_lobatto01(n):
    """Gauss-Lobatto nodes on [0,1] in DEScending order (1 first, 0 last): the order of the
    reference's lobatto::nodes tables, which its Legendre-to-Lobatto projector follows."""
    N = n - 1
    xs = [mp.mpf(1), mp.mpf(-1)]
    for k in range(1, N):
        # interior nodes: roots of P'_N, Newton from the Chebyshev-Gauss-Lobatto points
        x = mp.cos(mp.pi * k / N)
        for _ in range(100):
            p0, p1 = mp.mpf(1), x
            for j in range(2, N + 1):
                p0, p1 = p1, ((2 * j - 1) * x * p1 - (j - 1) * p0) / j
            dp = N * (x * p1 - p0) / (x * x - 1)               # P'_N
            d2p = (2 * x * dp - N * (N + 1) * p1) / (1 - x * x)  # P''_N (Legendre ODE)
            dx = dp / d2p
            x -= dx
            if abs(dx) < mp.mpf(10) ** (-45):
                break
        xs.append(x)
    return sorted(((x + 1) / 2 for x in xs), reverse=True)


def amr_limiter_operators(order):
    """Projectors between mesh levels and onto the limiter's finite-volume subcells:

    * fine[j][k][m] = phi_k((j + x_m) / 3): coarse basis function k at the fine node m of the j-th
      third of the cell (3:1 refinement), the single-level prolongation (3d/amrRoutines.cpph);
    * dg2fv[k][i] = sum_j w_j phi_k((i + x_j) / P): the mean of phi_k over subcell i of P = 2N+1;
    * fv2dg[i][k]: the least-squares DG reconstruction from the P subcell means under the constraint
      that the DG cell mean equals the subcell mean (Dumbser et al., J. Comput. Phys. 278 (2014));
      the saddle-point system is set up as LimiterProjectionMatrices.h:216-262 does;
    * leg2lob[k][i] = phi_k(lobatto node i) (lobatto nodes descending).
    """
    n = order + 1
    P = 2 * order + 1
    x, w = gauss_legendre01(n)
    fine = [[[basis(x, (j + x[m]) / 3)[0][k] for m in range(n)] for k in range(n)] for j in range(3)]
    dg2fv = [[mp.mpf(0)] * P for _ in range(n)]
    for i in range(P):
        for j in range(n):
            phi, _ = basis(x, (i + x[j]) / P)
            for k in range(n):
                dg2fv[k][i] += w[j] * phi[k]
    M = mp.matrix(n + 1, n + 1)
    for i in range(n):
        for j in range(n):
            M[i, j] = sum(2 * dg2fv[i][k] * dg2fv[j][k] for k in range(P))
        M[i, n] = w[i]
        M[n, i] = -w[i]
    iM = M ** -1
    rhs = [[2 * dg2fv[j][i] for j in range(n)] + [mp.mpf(1) / P] for i in range(P)]
    fv2dg = [[sum(iM[k, j] * rhs[i][k] for k in range(n + 1)) for j in range(n)] for i in range(P)]
    lob = gauss_lobatto01(n)
    leg2lob = [[basis(x, lob[i])[0][k] for i in range(n)] for k in range(n)]
    return dict(fine=fine, dg2fv=dg2fv, fv2dg=fv2dg, leg2lob=leg2lob, lobatto=lob, P=P)


def fmt(v):
    return repr(float(v)) if float(v) != 0.0 else "0.0"


def main():
    out = []
    out.append("// Generated by exahype-engine_b200/gen_tables.py -- do not edit.")
    out.append("// 1D Gauss-Legendre ADER-DG operators on [0,1] (see the generator for definitions),")
    out.append("// as __constant__ arrays with a per-order accessor. Loops over these tables are fully")
    out.append("// unrolled in the kernels, so every access is a uniform constant-bank operand.")
    out.append("#pragma once")
    out.append("namespace exa {")
    out.append("template <int N> struct GL;")
    for o in range(1, MAX_ORDER + 1):
        n = o + 1
        t = operators(o)
        for k in ("nodes", "weights", "F0", "F1"):
            out.append("static __constant__ double c_%s_%d[%d] = {%s};" % (k, o, n, ", ".join(fmt(v) for v in t[k])))
        for k in ("Kxi", "iK1", "dudx"):
            rows = ["{%s}" % ", ".join(fmt(v) for v in r) for r in t[k]]
            out.append("static __constant__ double c_%s_%d[%d][%d] = {%s};" % (k, o, n, n, ", ".join(rows)))
        for k in ("Kxi", "iK1"):
            rows = ["{%s}" % ", ".join(fmt(v) + "f" if "e" in fmt(v) or "." in fmt(v) else fmt(v) for v in
                                  (float(x) for x in r)) for r in t[k]]
            out.append("static __constant__ float c_%sf_%d[%d][%d] = {%s};" % (k, o, n, n, ", ".join(rows)))
        out.append("template <> struct GL<%d> {" % o)
        out.append("  static constexpr int n = %d;" % n)
        for k in ("nodes", "weights", "F0", "F1"):
            out.append("  static __device__ __forceinline__ double %s(int i) { return c_%s_%d[i]; }" % (k, k, o))
        for k in ("Kxi", "iK1", "dudx"):
            out.append("  static __device__ __forceinline__ double %s(int i, int j) { return c_%s_%d[i][j]; }" % (k, k, o))
        out.append("  static __device__ __forceinline__ float Kxif(int i, int j) { return c_Kxif_%d[i][j]; }" % o)
        out.append("  static __device__ __forceinline__ float iK1f(int i, int j) { return c_iK1f_%d[i][j]; }" % o)
        out.append("};")
    # host copies of the quadrature (exa_quadrature), for glue code that evaluates user hooks
    out.append("// host-side quadrature nodes and weights, [order][node] (zero-padded to 10 entries)")
    rows_n, rows_w = [], []
    for o in range(1, MAX_ORDER + 1):
        t = operators(o)
        pad = [0.0] * (MAX_ORDER + 1 - (o + 1))
        rows_n.append("{%s}" % ", ".join(fmt(v) for v in list(t["nodes"]) + pad))
        rows_w.append("{%s}" % ", ".join(fmt(v) for v in list(t["weights"]) + pad))
    out.append("static const double h_nodes[%d][%d] = {%s};" % (MAX_ORDER, MAX_ORDER + 1, ", ".join(rows_n)))
    out.append("static const double h_weights[%d][%d] = {%s};" % (MAX_ORDER, MAX_ORDER + 1, ", ".join(rows_w)))
    out.append("}  // namespace exa")
    path = os.path.join(HERE, "csrc", "exa_tables.cuh")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
    print("wrote", path)
    write_amr_limiter_tables()


def write_amr_limiter_tables():
    out = []
    out.append("// Generated by exahype-engine_b200/gen_tables.py -- do not edit.")
    out.append("// Mesh-level and limiter projectors on [0,1] (amr_limiter_operators in the generator):")
    out.append("// fine[j][k][m], dg2fv[k][i], fv2dg[i][k], leg2lob[k][i], per order, with P = 2N+1 subcells.")
    out.append("#pragma once")
    out.append("namespace exa {")
    out.append("template <int N> struct AmrT;")
    hosts = []
    for o in range(1, MAX_ORDER + 1):
        n = o + 1
        t = amr_limiter_operators(o)
        P = t["P"]
        fine = ", ".join("{%s}" % ", ".join("{%s}" % ", ".join(fmt(v) for v in row) for row in blk) for blk in t["fine"])
        out.append("static __constant__ double c_fine_%d[3][%d][%d] = {%s};" % (o, n, n, fine))
        for k, (r, c) in (("dg2fv", (n, P)), ("fv2dg", (P, n)), ("leg2lob", (n, n))):
            rows = ", ".join("{%s}" % ", ".join(fmt(v) for v in row) for row in t[k])
            out.append("static __constant__ double c_%s_%d[%d][%d] = {%s};" % (k, o, r, c, rows))
        out.append("template <> struct AmrT<%d> {" % o)
        out.append("  static constexpr int n = %d, P = %d;" % (n, P))
        out.append("  static __device__ __forceinline__ double fine(int j, int k, int m) { return c_fine_%d[j][k][m]; }" % o)
        out.append("  static __device__ __forceinline__ double dg2fv(int k, int i) { return c_dg2fv_%d[k][i]; }" % o)
        out.append("  static __device__ __forceinline__ double fv2dg(int i, int k) { return c_fv2dg_%d[i][k]; }" % o)
        out.append("  static __device__ __forceinline__ double leg2lob(int k, int i) { return c_leg2lob_%d[k][i]; }" % o)
        out.append("};")
        flat = [v for blk in t["fine"] for row in blk for v in row] + [v for row in t["dg2fv"] for v in row] + \
            [v for row in t["fv2dg"] for v in row] + [v for row in t["leg2lob"] for v in row]
        hosts.append("static const double h_amr_lim_%d[%d] = {%s};" % (o, len(flat), ", ".join(fmt(v) for v in flat)))
    out.append("// host copies, per order: fine (3 n n), dg2fv (n P), fv2dg (P n), leg2lob (n n), concatenated")
    out.extend(hosts)
    out.append("static const double* const h_amr_lim[%d] = {nullptr, %s};" % (
        MAX_ORDER + 1, ", ".join("h_amr_lim_%d" % o for o in range(1, MAX_ORDER + 1))))
    out.append("}  // namespace exa")
    path = os.path.join(HERE, "csrc", "exa_amr_tables.cuh")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
    print("wrote", path)


if __name__ == "__main__":
    main()
