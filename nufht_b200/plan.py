"""Device-resident plan on CUDA tensors (the library's extension API, Part 2 of the C ABI)."""
import ctypes
import math

import numpy as np

from . import _lib as L


def _host_f64(a):
    try:
        import torch
        if isinstance(a, torch.Tensor):
            a = a.detach().to("cpu", torch.float64).numpy()
    except ImportError:  # pragma: no cover
        pass
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


class DevicePlan:
    """g = H c for fixed (nu, r, k, tol) on one GPU.

    r (m sources) and k (n targets) must be finite, non-negative and non-decreasing.
    Planning (box partition, work lists, FFT plans) happens once; each call runs the
    transform on the current torch stream.

    mixed: False (FP64), True (asymptotic boxes in FP32 where the planner's worst-case FP32
    error bound is within tol / 4, FP64 elsewhere) or "averaged" (FP32 for tol >= 1e-9
    regardless of that bound: within tol when each column's mass is spread over many
    sources, up to stats()[14] * ||c||_1 for a column concentrated on one source).
    info()["mixed"] says whether the asymptotic boxes run in FP32.
    """

    def __init__(self, nu, r, k, tol=1e-8, *, mixed=False, extended_tables=False, device=None,
                 max_levels=0, min_dim_prod=10000, z_split=math.nan, K_asy=0, K_loc=0):
        import torch
        lib = L.lib()
        self.nu = float(nu)
        self.tol = float(tol)
        rh, kh = _host_f64(r), _host_f64(k)
        self.m, self.n = rh.shape[0], kh.shape[0]
        if device is None:
            device = torch.cuda.current_device()
        self.device = torch.device("cuda", int(device) if not isinstance(device, torch.device) else device.index or 0)
        if mixed not in (False, True, "averaged"):
            raise ValueError("mixed must be False, True or 'averaged'")
        flags = ((L.NUFHT_B200_MIXED_AVERAGED if mixed == "averaged" else L.NUFHT_B200_MIXED if mixed else 0)
                 | (L.NUFHT_B200_EXTENDED_TABLES if extended_tables else 0))
        opt = L.options(tol=self.tol, max_levels=max_levels, min_dim_prod=min_dim_prod, z_split=z_split,
                        K_asy=K_asy, K_loc=K_loc)
        h = ctypes.c_void_p()
        rc = lib.nufht_b200_plan_create(ctypes.byref(h), self.nu, L.dptr(rh), self.m, L.dptr(kh), self.n,
                                        ctypes.byref(opt), flags, self.device.index)
        if rc != 0:
            raise RuntimeError("nufht_b200_plan_create failed (%d): %s" % (rc, L.strerror(rc)))
        self._h = h
        self.mixed = mixed

    def stats(self):
        """Work counts of the plan, its FP32 error model and its planning time
        (nufht_b200_plan_stats, 21 values)."""
        st = np.zeros(21)
        L.lib().nufht_b200_plan_stats(self._h, st.ctypes.data_as(L.c_double_p), 21)
        return st

    def info(self):
        inf = L.NufhtB200Info()
        L.lib().nufht_b200_plan_info(self._h, ctypes.byref(inf))
        return {f: getattr(inf, f) for f, _ in inf._fields_}

    def buffers(self):
        """(current asymptotic-grid workspace address, older workspace buffers kept for batch
        graphs that recorded them, number of batches pinning the plan)."""
        g = ctypes.c_void_p()
        ret = ctypes.c_int()
        pins = ctypes.c_int()
        L.lib().nufht_b200_plan_buffers(self._h, ctypes.byref(g), ctypes.byref(ret), ctypes.byref(pins))
        return g.value, ret.value, pins.value

    def boxes(self):
        lib = L.lib()
        tot = lib.nufht_b200_plan_boxes(self._h, None, 0)
        buf = np.zeros(4 * max(tot, 1), dtype=np.int32)
        lib.nufht_b200_plan_boxes(self._h, buf.ctypes.data_as(L.c_int_p), tot)
        inf = self.info()
        b = buf[:4 * tot].reshape(-1, 4)
        return b  # loc, then asy, then dir (planner order)

    def execute_columns(self, c_cols, out_cols=None, stream=None):
        """c_cols: CUDA float64 tensor (B, m) contiguous (column t = row t).  Returns (B, n)."""
        import torch
        assert c_cols.is_cuda and c_cols.dtype == torch.float64 and c_cols.is_contiguous()
        B = c_cols.shape[0]
        assert c_cols.shape[1] == self.m
        if out_cols is None:
            out_cols = torch.empty((B, self.n), dtype=torch.float64, device=c_cols.device)
        st = stream if stream is not None else torch.cuda.current_stream(c_cols.device)
        rc = L.lib().nufht_b200_execute(self._h, ctypes.c_void_p(c_cols.data_ptr()), self.m,
                                        ctypes.c_void_p(out_cols.data_ptr()), self.n, B,
                                        ctypes.c_void_p(st.cuda_stream))
        if rc != 0:
            raise RuntimeError("nufht_b200_execute failed (%d): %s" % (rc, L.strerror(rc)))
        return out_cols

    def __call__(self, c):
        """c: (m,) or (m, B) tensor (any device); returns (n,) or (n, B) on this plan's GPU."""
        import torch
        c = torch.as_tensor(c)
        squeeze = c.dim() == 1
        cc = c.reshape(self.m, -1).t().to(self.device, torch.float64).contiguous()
        g = self.execute_columns(cc)
        g = g.t()
        return g[:, 0] if squeeze else g

    def close(self):
        if getattr(self, "_h", None):
            L.lib().nufht_b200_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
