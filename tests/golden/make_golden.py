"""Generate the committed golden fixtures under tests/golden/.

Run where the reference checkout is present (--ref, or the EXAHYPE_REF environment variable) and the built
checker library oracle/_ref (``make -C oracle ref``):

    python tests/golden/make_golden.py [--ref PATH_TO_EXAHYPE_CHECKOUT]

Outputs
-------
generic_euler_{2d,3d}.npz
    Every array of the reference's own known-answer file
    ExaHyPE/exahype/tests/kernels/testdata/generic_euler_testdata.cpp, keyed
    ``<namespace>.<name>`` (e.g. ``testRiemannSolverNonlinear.FL``), parsed as text.
gl_tables.npz
    The reference's DG operator tables (weights, nodes, Kxi, iK1, dudx, FCoeff for orders
    0..9) parsed from ExaHyPE/kernels/generated/GaussLegendreBasis.csnippet.
limiter_{2d,3d}.npz
    Every array of the reference's limiter known-answer file
    ExaHyPE/exahype/tests/kernels/testdata/limiter_testdata.cpp (N = 3, nVar = 5, P = 7 subcells:
    luh -> subcell means, subcell means -> luh, luh -> Gauss-Lobatto values), parsed as text.
picard_euler3d_o3.npz, picard_euler2d_o3.npz
    Outputs of the reference's generic kernels (through oracle/_ref) on seeded NON-constant
    cells, which exercise the Picard iteration that the known-answer file leaves trivial.
"""
import argparse
import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

_ARRAY = re.compile(r"(?:const\s+)?double\s+(\w+)\s*\[\s*(\d+)\s*\]\s*=?\s*\{(.*?)\}\s*;", re.S)


def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def parse_testdata(path):
    """Return {'2d': {key: array}, '3d': {key: array}} from a known-answer file of the reference
    (generic_euler_testdata.cpp, limiter_testdata.cpp)."""
    raw = open(path).read()
    out = {"2d": {}, "3d": {}}
    for dim, tag in (("2d", "Dim2"), ("3d", "Dim3")):
        m = re.search(r"#ifdef\s+%s(.*?)#endif" % tag, raw, re.S)
        section = _strip_comments(m.group(1))
        # walk the namespaces; array bodies are consumed whole, so a lone '}' closes a namespace
        ns = []
        tokens = re.finditer(r"(?P<arr>(?:const\s+)?double\s+\w+\s*\[\s*\d+\s*\]\s*=?\s*\{.*?\}\s*;)|"
                             r"namespace\s+(?P<ns>\w+)\s*\{|(?P<close>\})", section, re.S)
        for t in tokens:
            if t.group("ns"):
                ns.append(t.group("ns"))
            elif t.group("close"):
                if ns:
                    ns.pop()
            else:
                a = _ARRAY.match(t.group("arr").strip())
                name, n, body = a.group(1), int(a.group(2)), a.group(3)
                vals = [float(x) for x in body.replace("\n", " ").split(",") if x.strip()]
                arr = np.zeros(n)
                arr[: len(vals)] = vals
                out[dim]["%s.%s" % (ns[-1] if ns else "", name)] = arr
    return out


def parse_gl_tables(path, max_order=9):
    text = open(path).read()
    tabs = {}

    def vec(name):
        m = re.search(r"double kernels::legendre::%s\[[^\]]*\]=\{(.*?)\};" % re.escape(name), text, re.S)
        return np.array([float(x) for x in m.group(1).replace("\n", " ").split(",") if x.strip()])

    for o in range(max_order + 1):
        n = o + 1
        tabs["weights_%d" % o] = vec("weights_%d" % o)
        tabs["nodes_%d" % o] = vec("nodes_%d" % o)
        for mat in ("Kxi", "iK1", "dudx"):
            tabs["%s_%d" % (mat, o)] = np.stack([vec("%s_%d_%d" % (mat, o, r)) for r in range(n)])
        tabs["FCoeff0_%d" % o] = vec("FCoeff_0_%d" % o)
        tabs["FCoeff1_%d" % o] = vec("FCoeff_1_%d" % o)
    return tabs


def _ref(dim):
    lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libexaref%dd.so" % dim))
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def euler_state(rng, shape_nodes, amp=0.1):
    """A smooth, strictly admissible Euler state per node: rho, rho*u, E (p > 0)."""
    nn = shape_nodes
    rho = 1.0 + amp * rng.uniform(-1, 1, nn)
    u = 0.3 * rng.uniform(-1, 1, (nn, 3))
    p = 1.0 + amp * rng.uniform(-1, 1, nn)
    Q = np.zeros((nn, 5))
    Q[:, 0] = rho
    Q[:, 1:4] = rho[:, None] * u
    Q[:, 4] = p / 0.4 + 0.5 * rho * (u ** 2).sum(1)
    return Q


def picard_fixture(dim, order, seed=7, ncase=4):
    lib = _ref(dim)
    name = "exaref%dd_euler_o%d_p0" % (dim, order)
    n = order + 1
    nd = n ** dim
    nf = n ** (dim - 1)
    v = D = 5
    rng = np.random.default_rng(seed)
    fx = {}
    pred = getattr(lib, name + "_predictor")
    pred.restype = ctypes.c_int
    vol = getattr(lib, name + "_volume")
    dtf = getattr(lib, name + "_dt")
    dtf.restype = ctypes.c_double
    for c in range(ncase):
        # perturbation amplitude grows with the case index so Picard counts differ
        luh = euler_state(rng, nd, amp=0.02 * (c + 1)).reshape(-1)
        if dim == 2:
            luh = luh.reshape(nd, 5)
            luh[:, 3] = 0.0  # the 2D system carries an unused z-momentum
            luh = luh.reshape(-1)
        dx = np.array([0.05, 0.04, 0.03][:dim] + [0.0] * (3 - dim))
        centre = np.array([0.3, 0.6, 0.2])
        dt = float(dtf(_p(luh), _p(dx)))
        lQi = np.zeros(D * nd * n)
        rhs = np.zeros(D * nd * n)
        lFi = np.zeros((dim + 1) * v * nd * n)
        gradQ = np.zeros(dim * v * nd)
        lQhi = np.zeros(D * nd)
        lFhi = np.zeros((dim + 1) * v * nd)
        lQhbnd = np.zeros(2 * dim * nf * D)
        lFhbnd = np.zeros(2 * dim * nf * v)
        it = pred(_p(luh), _p(centre), _p(dx), ctypes.c_double(0.0), ctypes.c_double(dt), _p(lQi), _p(rhs),
                  _p(lFi), _p(gradQ), _p(lQhi), _p(lFhi), _p(lQhbnd), _p(lFhbnd))
        lduh = np.zeros(v * nd)
        vol(_p(lduh), _p(lFhi), _p(dx))
        for k, a in dict(luh=luh, dx=dx, dt=np.array([dt]), iters=np.array([it]), lQi=lQi, lQhi=lQhi,
                         lFhi=lFhi, lQhbnd=lQhbnd, lFhbnd=lFhbnd, lduh=lduh).items():
            fx["case%d.%s" % (c, k)] = a
    fx["ncase"] = np.array([ncase])
    return fx


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("EXAHYPE_REF", "/root/reference"))
    args = ap.parse_args()
    td = parse_testdata(os.path.join(args.ref, "ExaHyPE/exahype/tests/kernels/testdata/generic_euler_testdata.cpp"))
    for dim in ("2d", "3d"):
        np.savez_compressed(os.path.join(HERE, "generic_euler_%s.npz" % dim), **td[dim])
        print(dim, len(td[dim]), "arrays")
    lt = parse_testdata(os.path.join(args.ref, "ExaHyPE/exahype/tests/kernels/testdata/limiter_testdata.cpp"))
    for dim in ("2d", "3d"):
        np.savez_compressed(os.path.join(HERE, "limiter_%s.npz" % dim), **lt[dim])
        print("limiter", dim, len(lt[dim]), "arrays")
    gl = parse_gl_tables(os.path.join(args.ref, "ExaHyPE/kernels/generated/GaussLegendreBasis.csnippet"))
    np.savez_compressed(os.path.join(HERE, "gl_tables.npz"), **gl)
    print("gl tables", len(gl))
    np.savez_compressed(os.path.join(HERE, "picard_euler3d_o3.npz"), **picard_fixture(3, 3))
    np.savez_compressed(os.path.join(HERE, "picard_euler2d_o3.npz"), **picard_fixture(2, 3))
    print("picard fixtures written")


if __name__ == "__main__":
    main()
