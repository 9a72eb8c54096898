"""Drop-in for the reference's Python extension module `_pynufht` (src/_pynufht.c).

Same three functions, argument meaning, result layout and exceptions:

  nufht(nu, rs, cs, ws, tol=1e-8)            -> ndarray (n,)
  nufht_batch(nu, rs, cs, ws, tol=1e-8)      -> ndarray (n, batch), C order
  nufht_batch_loop(nu, rs, cs, ws, tol=1e-8) -> ndarray (n, batch), one transform per column

Each call runs the transform on the GPU through the C ABI of libnufht_b200.so.  The
reference plans on the CPU per call (src/_pynufht.c:186); `nufht_batch` here keeps the last
few plans (keyed by order, tolerance and the grids' contents) and reuses them.
"""
import ctypes
import hashlib
import os

import numpy as np

from . import _lib as L

__all__ = ["nufht", "nufht_batch", "nufht_batch_loop"]


def _vec(a):
    return L.as_f64(a, "C").ravel() if np.ndim(a) != 1 else L.as_f64(a, "C")


def nufht(nu, rs, cs, ws, tol=1e-8):
    """Single transform via the C entry point nufht() (src/_pynufht.c:17-62)."""
    lib = L.lib()
    rs = _vec(rs)
    ws = _vec(ws)
    cs = L.as_f64(cs, "C")
    m, n = rs.shape[0], ws.shape[0]
    opt = L.options(tol=float(tol))
    out = lib.nufht(float(nu), L.dptr(rs), m, L.dptr(cs), L.dptr(ws), n, ctypes.byref(opt))
    if not out:
        raise RuntimeError("nufht returned NULL")
    try:
        res = np.ctypeslib.as_array(ctypes.cast(out, ctypes.POINTER(ctypes.c_double)), shape=(n,)).copy()
    finally:
        ctypes.CDLL(None).free(ctypes.c_void_p(out))
    return res


def _check_batch(rs, cs):
    cs = np.asarray(cs, dtype=np.float64)
    if cs.ndim != 2:
        raise ValueError("cs must be 2-D array with shape (m, batch)")
    if cs.shape[0] != rs.shape[0]:
        raise ValueError("cs first dimension must match rs length")
    return cs


class _PlanCache:
    """The last few plans, keyed by (nu, tol, grids).  The reference plans on every call
    (src/_pynufht.c:186); repeated calls on the same grids here reuse the host plan and its
    device state (work lists, FFT plans, workspace).  The grids are kept alive with the plan,
    which borrows them."""

    def __init__(self, size=4):
        self.size = size
        self.entries = []  # (key, plan, rs, ws), most recent last

    @staticmethod
    def key(nu, tol, rs, ws):
        h = hashlib.blake2b(digest_size=16)
        h.update(rs.tobytes())
        h.update(ws.tobytes())
        # the precision switch of the reference entry points is read when a plan first runs
        return (float(nu), float(tol), rs.shape[0], ws.shape[0], h.digest(),
                os.environ.get("NUFHT_B200_PRECISION", ""))

    def get(self, nu, tol, rs, ws):
        k = self.key(nu, tol, rs, ws)
        for q, (kk, plan, r, w) in enumerate(self.entries):
            if kk == k:
                self.entries.append(self.entries.pop(q))
                return plan
        lib = L.lib()
        opt = L.options(tol=float(tol))
        plan = L.NufhtPlan()
        rs = rs.copy()
        ws = ws.copy()
        if lib.nufht_plan_init(ctypes.byref(plan), float(nu), L.dptr(rs), rs.shape[0], L.dptr(ws), ws.shape[0],
                               ctypes.byref(opt)) != 0:
            lib.nufht_plan_free(ctypes.byref(plan))
            raise RuntimeError("nufht_plan_init failed")
        self.entries.append((k, plan, rs, ws))
        while len(self.entries) > self.size:
            _, old, _, _ = self.entries.pop(0)
            lib.nufht_plan_free(ctypes.byref(old))
        return plan

    def clear(self):
        lib = L.lib()
        for _, plan, _, _ in self.entries:
            lib.nufht_plan_free(ctypes.byref(plan))
        self.entries = []


_plans = _PlanCache()


def clear_plan_cache():
    """Release the cached plans (and their device memory)."""
    _plans.clear()


def nufht_batch(nu, rs, cs, ws, tol=1e-8):
    """Batched transform through nufht_plan_init / nufht_batch (src/_pynufht.c:144-239).

    Same arguments, C-order (n, batch) result and exceptions as the reference.  The reference
    copies cs to Fortran order and transposes g back on the host (src/_pynufht.c:156,
    222-237); here C-order or Fortran-order cs is read as it is and the C-order result is
    written directly (nufht_b200_batch_layout transposes on the GPU)."""
    lib = L.lib()
    rs = _vec(rs)
    ws = _vec(ws)
    cs = _check_batch(rs, cs)
    m, n, batch = rs.shape[0], ws.shape[0], cs.shape[1]
    if cs.flags.c_contiguous:
        c_row, ld_cs = 1, batch
    elif cs.flags.f_contiguous:
        c_row, ld_cs = 0, m
    else:
        cs = np.ascontiguousarray(cs)
        c_row, ld_cs = 1, batch
    plan = _plans.get(nu, tol, rs, ws)
    gs = np.empty((n, batch), dtype=np.float64)  # C order, as the reference returns
    ret = lib.nufht_b200_batch_layout(ctypes.byref(plan), L.dptr(cs), c_row, ld_cs, L.dptr(gs), 1, batch, batch)
    if ret != 0:
        raise RuntimeError("nufht_batch returned %d" % ret)
    return gs


def nufht_batch_loop(nu, rs, cs, ws, tol=1e-8):
    """Batch by looping single transforms over the columns (src/_pynufht.c:64-142)."""
    rs = _vec(rs)
    ws = _vec(ws)
    cs = _check_batch(rs, cs)
    out = np.empty((ws.shape[0], cs.shape[1]), dtype=np.float64)
    for b in range(cs.shape[1]):
        out[:, b] = nufht(nu, rs, np.ascontiguousarray(cs[:, b]), ws, tol)
    return out
