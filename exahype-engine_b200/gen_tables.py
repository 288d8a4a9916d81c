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


if __name__ == "__main__":
    main()
