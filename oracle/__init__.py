"""CPU oracle for the batched NUFHT -- TEST INFRASTRUCTURE ONLY.

Loaded only by tests/, __graft_entry__.smoke() and bench.py (CPU-baseline and reference
arms) as the checker; the product library never imports it.  Wraps:

  liboracle.so          plain-C restatement of the reference (nufht_oracle.c)
  _ref/libnufht_ref.so  the reference's own driver/planner compiled unchanged, linked with the
                        oracle's evaluators (present only where the reference tree was available
                        at build time)
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libnufht_ref.so")
TABLES = os.path.join(ROOT, "nufht_b200", "data", "nufht_tables.cache")

T3_EXACT, T3_NUFFT = 0, 1
_o = None
_ref = None

vp = ctypes.c_void_p
cd = ctypes.c_double
ci = ctypes.c_int


def _p(a):
    return a.ctypes.data_as(vp)


def lib():
    global _o
    if _o is None:
        from . import build as _b
        _b.build()  # rebuilds only when the sources are newer than the library
        o = ctypes.CDLL(LIB_PATH)
        o.oracle_load_tables.argtypes = [ctypes.c_char_p]
        o.oracle_plan_params.argtypes = [cd, cd, cd, ci, ci, vp, vp, vp, vp]
        o.oracle_generate_boxes.argtypes = [vp, ci, vp, ci, cd, ci, ci, ci, vp, vp, ctypes.c_long]
        o.oracle_generate_boxes.restype = ctypes.c_long
        o.oracle_nufht_batch.argtypes = [cd, vp, ci, vp, ci, vp, ci, vp, ci, ci, cd, ci, ci, cd, ci, ci, ci]
        o.oracle_direct_sum.argtypes = [cd, vp, ci, vp, vp, ci, ci, vp, ci, vp]
        o.oracle_set_type3_mode.argtypes = [ci]
        o.oracle_set_threads.argtypes = [ci]
        o.oracle_besselj.argtypes = [cd, cd]
        o.oracle_besselj.restype = cd
        o.oracle_type3.argtypes = [ci, ci, vp, vp, cd, ci, vp, vp]
        rc = o.oracle_load_tables(TABLES.encode())
        if rc != 0:
            raise RuntimeError("oracle: cannot load tables from %s (%d)" % (TABLES, rc))
        _o = o
    return _o


def set_threads(n):
    lib().oracle_set_threads(int(n))


def plan_params(nu, tol, z_split=math.nan, K_asy=0, K_loc=0):
    z = np.zeros(1)
    ka = np.zeros(1, np.int32)
    kl = np.zeros(1, np.int32)
    coef = np.zeros(64)
    rc = lib().oracle_plan_params(nu, tol, z_split, K_asy, K_loc, _p(z), _p(ka), _p(kl), _p(coef))
    return rc, float(z[0]), int(ka[0]), int(kl[0]), coef


def boxes(rs, ws, z_split, max_levels=0, min_dim_prod=10000, K_loc=0):
    rs = np.ascontiguousarray(rs, np.float64)
    ws = np.ascontiguousarray(ws, np.float64)
    cnt = np.zeros(3, np.int64)
    tot = lib().oracle_generate_boxes(_p(rs), len(rs), _p(ws), len(ws), z_split, max_levels, min_dim_prod,
                                      K_loc, _p(cnt), None, 0)
    out = np.zeros((max(tot, 1), 4), np.int32)
    lib().oracle_generate_boxes(_p(rs), len(rs), _p(ws), len(ws), z_split, max_levels, min_dim_prod, K_loc,
                                _p(cnt), _p(out), tot)
    a, b = cnt[0], cnt[0] + cnt[1]
    return out[:a].astype(np.int64), out[a:b].astype(np.int64), out[b:tot].astype(np.int64)


def nufht_batch(nu, rs, ws, cs, tol=1e-8, mode=T3_EXACT, faithful=False, max_levels=0, min_dim_prod=10000,
                z_split=math.nan, K_asy=0, K_loc=0):
    """g (n, B) = oracle transform of cs (m, B)."""
    o = lib()
    o.oracle_set_type3_mode(mode)
    rs = np.ascontiguousarray(rs, np.float64)
    ws = np.ascontiguousarray(ws, np.float64)
    cs = np.asfortranarray(np.asarray(cs, np.float64).reshape(len(rs), -1))
    B = cs.shape[1]
    gs = np.zeros((len(ws), B), order="F")
    rc = o.oracle_nufht_batch(nu, _p(rs), len(rs), _p(ws), len(ws), _p(cs), len(rs), _p(gs), len(ws), B, tol,
                              max_levels, min_dim_prod, z_split, K_asy, K_loc, 1 if faithful else 0)
    if rc != 0:
        raise RuntimeError("oracle_nufht_batch returned %d" % rc)
    return gs


def direct_sum(nu, rs, ws, cs, idx):
    """Exact FP64 sums g[idx, t] (Kahan-compensated) -- the ground truth."""
    rs = np.ascontiguousarray(rs, np.float64)
    ws = np.ascontiguousarray(ws, np.float64)
    cs = np.asfortranarray(np.asarray(cs, np.float64).reshape(len(rs), -1))
    idx = np.ascontiguousarray(idx, np.int64)
    out = np.zeros((len(idx), cs.shape[1]), order="F")
    lib().oracle_direct_sum(nu, _p(rs), len(rs), _p(ws), _p(cs), len(rs), cs.shape[1], _p(idx), len(idx), _p(out))
    return out


def besselj(nu, x):
    f = lib().oracle_besselj
    return np.array([f(float(nu), float(v)) for v in np.ravel(x)])


def type3(x, c, s, eps=1e-12, mode=T3_NUFFT):
    """f[t, k] = sum_j c[t, j] exp(i s_k x_j); c complex (ntr, nj)."""
    o = lib()
    o.oracle_set_type3_mode(mode)
    x = np.ascontiguousarray(x, np.float64)
    s = np.ascontiguousarray(s, np.float64)
    c = np.ascontiguousarray(np.atleast_2d(c), np.complex128)
    f = np.zeros((c.shape[0], len(s)), np.complex128)
    rc = o.oracle_type3(c.shape[0], len(x), _p(x), _p(c), eps, len(s), _p(s), _p(f))
    if rc != 0:
        raise RuntimeError("oracle_type3 returned %d" % rc)
    return f


def ref_available():
    return os.path.exists(REF_PATH)


def ref():
    """The reference's own driver/planner (compiled unchanged) over the oracle's evaluators."""
    global _ref
    if _ref is None:
        os.environ.setdefault("NUFHT_TABLE_CACHE", TABLES)
        import sys
        sys.path.insert(0, ROOT)
        from nufht_b200 import _lib as L
        r = ctypes.CDLL(REF_PATH)
        L._declare_ref = None
        for name, res, args in [
            ("nufht_default_options", L.NufhtOptions, []),
            ("nufht_plan_init", ci, [ctypes.POINTER(L.NufhtPlan), cd, vp, ci, vp, ci, ctypes.POINTER(L.NufhtOptions)]),
            ("nufht_plan_free", None, [ctypes.POINTER(L.NufhtPlan)]),
            ("nufht_batch", ci, [ctypes.POINTER(L.NufhtPlan), vp, ci, vp, ci, ci, vp]),
            ("generate_boxes", L.Boxes, [vp, ci, vp, ci, cd, ci, ci, ci]),
            ("boxes_free", None, [ctypes.POINTER(L.Boxes)]),
        ]:
            f = getattr(r, name)
            f.restype = res
            f.argtypes = args
        r.oracle_set_type3_mode.argtypes = [ci]
        r.oracle_set_threads.argtypes = [ci]
        _ref = r
    return _ref


def ref_nufht_batch(nu, rs, ws, cs, tol=1e-8, mode=T3_EXACT):
    """Reference nufht_plan_init + nufht_batch (its own control flow) on the oracle evaluators."""
    from nufht_b200 import _lib as L
    r = ref()
    r.oracle_set_type3_mode(mode)
    rs = np.ascontiguousarray(rs, np.float64)
    ws = np.ascontiguousarray(ws, np.float64)
    cs = np.asfortranarray(np.asarray(cs, np.float64).reshape(len(rs), -1))
    B = cs.shape[1]
    gs = np.zeros((len(ws), B), order="F")
    opt = r.nufht_default_options()
    opt.tol = tol
    plan = L.NufhtPlan()
    import contextlib
    rc = r.nufht_plan_init(ctypes.byref(plan), nu, _p(rs), len(rs), _p(ws), len(ws), ctypes.byref(opt))
    if rc != 0:
        raise RuntimeError("reference nufht_plan_init returned %d" % rc)
    try:
        rc = r.nufht_batch(ctypes.byref(plan), _p(cs), len(rs), _p(gs), len(ws), B, None)
        if rc != 0:
            raise RuntimeError("reference nufht_batch returned %d" % rc)
    finally:
        r.nufht_plan_free(ctypes.byref(plan))
    return gs


def ref_boxes(rs, ws, z_split, max_levels=0, min_dim_prod=10000, K_loc=0):
    from nufht_b200 import _lib as L
    r = ref()
    rs = np.ascontiguousarray(rs, np.float64)
    ws = np.ascontiguousarray(ws, np.float64)
    b = r.generate_boxes(_p(rs), len(rs), _p(ws), len(ws), z_split, max_levels, min_dim_prod, K_loc)
    out = L.boxes_to_array(b)
    r.boxes_free(ctypes.byref(b))
    return out
