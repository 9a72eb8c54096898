"""Differentiable NUFHT on CUDA tensors.

    g[i,t] = sum_j c[j,t] J_nu(k_i r_j)

Backward (hand-written, every term a transform of the same method on the GPU):
  dL/dc[j,t] = sum_i u[i,t] J_nu(k_i r_j)                     = (H_nu^T u)[j,t]
  dL/dr_j    = sum_t c[j,t] sum_i u[i,t] k_i J_nu'(k_i r_j)
             = sum_t c[j,t] (H_{nu-1}^T (k u) - H_{nu+1}^T (k u))[j,t] / 2
  dL/dk_i    = sum_t u[i,t] sum_j c[j,t] r_j J_nu'(k_i r_j)
             = sum_t u[i,t] (H_{nu-1} (r c) - H_{nu+1} (r c))[i,t] / 2
with u = dL/dg and J_nu' = (J_{nu-1} - J_{nu+1}) / 2; H^T is the transform with the roles
of r and k exchanged (sources k, targets r).  For nu = 0 the derivative is -J_1 (one
transform per gradient).  Half-integer orders below 1 use J_nu' = (nu/x) J_nu - J_{nu+1}:
the transform defines negative half-integer orders as J_|nu|, which is not J_{nu-1}.
"""
import torch

from .plan import DevicePlan


def _sorted(x):
    return bool(torch.all(x[1:] >= x[:-1])) if x.numel() > 1 else True


class HankelPlans:
    """Plans of the transforms the forward and backward passes need, for fixed grids.

    Each (order, direction) pair is planned on first use and kept, so repeated calls on the
    same r and k plan once."""

    def __init__(self, nu, r, k, tol=1e-8, mixed=False, extended_tables=False):
        self.nu, self.tol, self.mixed = float(nu), float(tol), mixed
        self.r = r.detach().to(torch.float64)
        self.k = k.detach().to(torch.float64)
        self.extended = bool(extended_tables)
        self._cache = {}

    def plan(self, order, adjoint):
        key = (float(order), bool(adjoint))
        if key not in self._cache:
            a, b = (self.k, self.r) if adjoint else (self.r, self.k)
            self._cache[key] = DevicePlan(order, a, b, self.tol, mixed=self.mixed,
                                          extended_tables=self.extended, device=a.device)
        return self._cache[key]

    def apply(self, order, adjoint, x):
        """x: (rows, B) float64 on the GPU -> (rows', B)."""
        p = self.plan(order, adjoint)
        return p.execute_columns(x.t().contiguous()).t()

    def close(self):
        for p in self._cache.values():
            p.close()
        self._cache.clear()


class NufhtFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, c, r, k, plans):
        g = plans.apply(plans.nu, False, c)
        ctx.save_for_backward(c, r, k)
        ctx.plans = plans
        return g

    @staticmethod
    def backward(ctx, u):
        c, r, k = ctx.saved_tensors
        P = ctx.plans
        nu = P.nu
        u = u.contiguous()
        dc = dr = dk = None
        symmetric = float(nu).is_integer() or nu >= 1.0
        Hu = None
        if ctx.needs_input_grad[0] or (ctx.needs_input_grad[1] and not symmetric):
            Hu = P.apply(nu, True, u)
        if ctx.needs_input_grad[0]:
            dc = Hu
        if ctx.needs_input_grad[1]:
            ku = u * k[:, None]
            if nu == 0.0:
                d = -P.apply(1.0, True, ku)
            elif symmetric:
                d = 0.5 * (P.apply(nu - 1.0, True, ku) - P.apply(nu + 1.0, True, ku))
            else:
                d = (nu / r)[:, None] * Hu - P.apply(nu + 1.0, True, ku)
            dr = (c * d).sum(dim=1)
        if ctx.needs_input_grad[2]:
            rc = c * r[:, None]
            if nu == 0.0:
                d = -P.apply(1.0, False, rc)
            elif symmetric:
                d = 0.5 * (P.apply(nu - 1.0, False, rc) - P.apply(nu + 1.0, False, rc))
            else:
                d = (nu / k)[:, None] * P.apply(nu, False, c) - P.apply(nu + 1.0, False, rc)
            dk = (u * d).sum(dim=1)
        return dc, dr, dk, None


def nufht(c, r, k, nu, tol=1e-8, mixed=False, plans=None):
    """Differentiable g = H c.  c: (m,) or (m, B); r: (m,), k: (n,) sorted, on one GPU.

    mixed: False, True or "averaged", as for DevicePlan.  Gradients flow to c, r and k.  Pass `plans` (a HankelPlans for the same grids) to reuse
    planning across calls with the same r and k."""
    squeeze = c.dim() == 1
    c2 = c.reshape(c.shape[0], -1).to(torch.float64)
    if not (_sorted(r) and _sorted(k)):
        raise ValueError("r and k must be sorted ascending")
    if plans is None:
        plans = HankelPlans(nu, r, k, tol, mixed)
    g = NufhtFunction.apply(c2, r.to(torch.float64), k.to(torch.float64), plans)
    return g[:, 0] if squeeze else g


class HankelTransform(torch.nn.Module):
    """Module wrapper: fixed order and tolerance; plans cached for the last grids seen.

    extended_tables fills the asymptotic table entry the reference leaves empty (K_asy = 10,
    reached by |nu| >= 35 at tol 1e-8)."""

    def __init__(self, nu, tol=1e-8, mixed=False, extended_tables=False):
        super().__init__()
        self.nu, self.tol, self.mixed = float(nu), float(tol), mixed
        self.extended = bool(extended_tables)
        self._plans = None
        self._key = None

    def forward(self, c, r, k):
        key = (r.data_ptr(), k.data_ptr(), r.numel(), k.numel(), r._version, k._version)
        if self._plans is None or key != self._key:
            self.release()
            self._plans = HankelPlans(self.nu, r, k, self.tol, self.mixed, self.extended)
            self._key = key
        return nufht(c, r, k, self.nu, self.tol, self.mixed, plans=self._plans)

    def release(self):
        """Free the cached plans and their device workspaces."""
        if self._plans is not None:
            self._plans.close()
        self._plans = None
        self._key = None
