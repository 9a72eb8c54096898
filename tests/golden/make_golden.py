"""Regenerate the golden fixtures in tests/golden/ (run in the build container).

  bessel_golden.npz  J_nu(x) from mpmath (30 digits) on a grid of orders and arguments
  tables_golden.npz  rows of the reference's shipped table cache (data/nufht_tables.cache)
  boxes_golden.npz   box partitions produced by the reference's own generate_boxes
                     (src/fast_hankel_nufht.c, compiled unchanged into oracle/_ref)
  e2e_golden.npz     outputs of the reference's own nufht_plan_init + nufht_batch control
                     flow (oracle/_ref) over the oracle's evaluators with exact type-3 sums

Usage: NUFHT_REFERENCE_DIR=<reference tree> python tests/golden/make_golden.py   (needs mpmath)
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF_DIR = os.environ.get("NUFHT_REFERENCE_DIR")
if __name__ == "__main__" and not REF_DIR:
    sys.exit("make_golden.py: set NUFHT_REFERENCE_DIR to the reference tree (it reads the table "
             "cache and builds the reference's planner from it)")


def grids(kind, m, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        r = np.sort(rng.uniform(0.0, 1.0, m)) * 200.0 + 1e-3
        k = np.sort(rng.uniform(0.0, 1.0, n)) * 200.0 + 1e-3
    elif kind == "loguniform":
        r = np.sort(10.0 ** rng.uniform(-3, 2, m))
        k = np.sort(10.0 ** rng.uniform(-2, 3, n))
    elif kind == "gl":
        x, _ = np.polynomial.legendre.leggauss(m)
        r = 25.0 * (x + 1.0)
        k = 10.0 * np.arange(1, n + 1) / n
    else:
        raise ValueError(kind)
    return r, k


BOX_CASES = [  # (kind, m, n, seed, nu, tol)
    ("gl", 10000, 200, 0, 0.0, 1e-8),
    ("uniform", 20000, 15000, 1, 0.0, 1e-8),
    ("uniform", 20000, 15000, 1, 0.0, 1e-6),
    ("uniform", 20000, 15000, 1, 0.0, 1e-10),
    ("loguniform", 12000, 9000, 2, 1.0, 1e-8),
    ("uniform", 5000, 7000, 3, 10.0, 1e-12),
    ("uniform", 3000, 3000, 4, 3.0, 1e-4),
]

E2E_CASES = [  # (name, kind, m, n, seed, nu, tol, B)
    ("nu0_uniform", "uniform", 1500, 1200, 11, 0.0, 1e-8, 3),
    ("nu1_loguniform", "loguniform", 1500, 1300, 12, 1.0, 1e-8, 2),
    ("nu2_uniform", "uniform", 1200, 1500, 13, 2.0, 1e-10, 2),
    ("nu3_uniform", "uniform", 1400, 1000, 14, 3.0, 1e-6, 3),
    ("nu10_uniform", "uniform", 1000, 1400, 15, 10.0, 1e-8, 2),
    ("num1_uniform", "uniform", 1300, 1100, 16, -1.0, 1e-8, 2),
    ("nu12_half", "uniform", 1100, 900, 17, 0.5, 1e-8, 2),
    ("direct_small", "uniform", 60, 90, 18, 2.0, 1e-8, 3),
    ("nu0_tol12", "uniform", 1200, 1200, 19, 0.0, 1e-12, 2),
]


def make_bessel():
    import mpmath as mp
    mp.mp.dps = 30
    rng = np.random.default_rng(5)
    orders, xs, vals = [], [], []
    for nu in [0, 1, 2, 3, 5, 10, 20, 35, 50, 100, 150, 200, 0.5, 1.5, 2.5, 3.5, 5.5, 9.5]:
        n = float(nu)
        x = np.concatenate([rng.uniform(0, 3 * n + 30, 60), np.logspace(-6, 6, 25),
                            n + rng.uniform(-3, 3, 15), [2 * math.sqrt(n + 1), max(n, 1e-3)]])
        x = x[x > 0]
        for v in x:
            orders.append(n)
            xs.append(v)
            vals.append(float(mp.besselj(n, mp.mpf(float(v)))))
    np.savez_compressed(os.path.join(HERE, "bessel_golden.npz"), nu=np.array(orders), x=np.array(xs),
                        j=np.array(vals))


def read_cache(path):
    f = open(path, "rb").read()
    off = 24
    coef = np.frombuffer(f, np.float64, 401 * 64, off).reshape(401, 64)
    off += 401 * 64 * 8
    z = np.frombuffer(f, np.float64, 401 * 32 * 16, off).reshape(401, 32, 16)
    off += 401 * 32 * 16 * 8
    kw = np.frombuffer(f, np.int32, 401 * 32 * 16, off).reshape(401, 32, 16)
    return coef, z, kw


def make_tables():
    coef, z, kw = read_cache(os.path.join(REF_DIR, "data", "nufht_tables.cache"))
    nus = np.array([0, 1, 2, 3, 10, 34, 35, 100, 200])
    np.savez_compressed(os.path.join(HERE, "tables_golden.npz"), nus=nus,
                        coef=np.stack([coef[2 * v] for v in nus] + [coef[2 * v + 1] for v in nus[:5]]),
                        coef_rows=np.array([2 * v for v in nus] + [2 * v + 1 for v in nus[:5]]),
                        z=np.stack([z[v, :12, :11] for v in nus]), kw=np.stack([kw[v, :12, :11] for v in nus]))


def make_boxes():
    import oracle
    out = {}
    for q, (kind, m, n, seed, nu, tol) in enumerate(BOX_CASES):
        r, k = grids(kind, m, n, seed)
        rc, z, ka, kl, _ = oracle.plan_params(nu, tol)
        loc, asy, dr = oracle.ref_boxes(r, k, z, 0, 10000, kl)
        out["case%d_meta" % q] = np.array([m, n, seed, nu, tol, z, ka, kl])
        out["case%d_kind" % q] = np.array(kind)
        out["case%d_loc" % q] = loc
        out["case%d_asy" % q] = asy
        out["case%d_dir" % q] = dr
    np.savez_compressed(os.path.join(HERE, "boxes_golden.npz"), **out)


def make_e2e():
    import oracle
    out = {}
    for name, kind, m, n, seed, nu, tol, B in E2E_CASES:
        r, k = grids(kind, m, n, seed)
        c = np.random.default_rng(seed + 100).standard_normal((m, B))
        g = oracle.ref_nufht_batch(nu, r, k, c, tol, mode=oracle.T3_EXACT)
        out[name + "_r"] = r
        out[name + "_k"] = k
        out[name + "_c"] = c
        out[name + "_g"] = g
        out[name + "_meta"] = np.array([nu, tol, B])
    np.savez_compressed(os.path.join(HERE, "e2e_golden.npz"), names=np.array([e[0] for e in E2E_CASES]), **out)


if __name__ == "__main__":
    make_tables()
    make_boxes()
    make_e2e()
    make_bessel()
    print("ok")
