"""Gradients of loss = ||H c - y||^2 with respect to c, r and k through
nufht_b200.torch_ops.nufht, against central finite differences (step 1e-6) of the FP64 loss
built from the oracle's direct sums, on random coordinates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _richardson(d1, d2):
    # Central differences D(h) = L' + a h^2 + O(h^4): (4 D(h) - D(2h)) / 3 cancels the h^2
    # term, which is large here (the third derivative in r_j grows like k^3).
    return (4.0 * d1 - d2) / 3.0


def _fd_r(orc, nu, r, k, c, y, g, j, h):
    """Central difference of L = ||g - y||^2 in r_j at steps h and 2h, Richardson-combined.
    Only source j moves, so g(r_j +- h) = g + p/m - b with p, m, b its moved / unmoved
    terms, and L+ - L- = sum (p - m) (2 (g - y) + p + m - 2 b), free of cancellation
    against L itself."""
    one = np.arange(len(k))
    b = orc.direct_sum(nu, r[j:j + 1], k, c[j:j + 1], one)
    d = []
    for hh in (h, 2 * h):
        rp, rm = r[j] + hh, r[j] - hh
        p = orc.direct_sum(nu, np.array([rp]), k, c[j:j + 1], one)
        m = orc.direct_sum(nu, np.array([rm]), k, c[j:j + 1], one)
        d.append(float(((p - m) * (2.0 * (g - y) + p + m - 2.0 * b)).sum()) / (rp - rm))
    return _richardson(*d)


def _fd_k(orc, nu, r, k, c, y, g, i, h):
    """As _fd_r for k_i: only row i of g moves."""
    b = orc.direct_sum(nu, r, k[i:i + 1], c, np.array([0]))[0]
    d = []
    for hh in (h, 2 * h):
        kp, km = k[i] + hh, k[i] - hh
        p = orc.direct_sum(nu, r, np.array([kp]), c, np.array([0]))[0]
        m = orc.direct_sum(nu, r, np.array([km]), c, np.array([0]))[0]
        d.append(float(((p - m) * (2.0 * (g[i] - y[i]) + p + m - 2.0 * b)).sum()) / (kp - km))
    return _richardson(*d)


@pytest.mark.parametrize("nu,rlo,rhi,klo,khi", [
    (1.0, -3, 2, -2, 3),        # the differentiation workload's ranges (log10), orders 0 and 2
    (0.0, -2, 1.5, -1, 2),      # J_0' = -J_1
    (0.5, 0.0, 1.5, 0.0, 1.2),  # half-integer: J' = (nu/x) J - J_{nu+1}
])
def test_gradients_vs_finite_differences(cuda, orc, nu, rlo, rhi, klo, khi):
    import torch
    from nufht_b200.torch_ops import nufht
    rng = np.random.default_rng(7)
    m, n, B = 1200, 1000, 3
    r = np.sort(10.0 ** rng.uniform(rlo, rhi, m))
    k = np.sort(10.0 ** rng.uniform(klo, khi, n))
    c0 = rng.standard_normal((m, B))
    y = orc.direct_sum(nu, r, k, c0, np.arange(n)) + 1e-3 * rng.standard_normal((n, B))
    c = c0 + 0.1 * rng.standard_normal((m, B))
    rt = torch.tensor(r, device=cuda, requires_grad=True)
    kt = torch.tensor(k, device=cuda, requires_grad=True)
    ct = torch.tensor(c, device=cuda, requires_grad=True)
    yt = torch.tensor(y, device=cuda)
    loss = ((nufht(ct, rt, kt, nu, tol=1e-12) - yt) ** 2).sum()
    loss.backward()
    g = orc.direct_sum(nu, r, k, c, np.arange(n))
    L0 = float(((g - y) ** 2).sum())
    assert abs(loss.item() - L0) <= 1e-9 * L0 + 1e-9
    h = 1e-6
    gr, gk, gc = rt.grad.cpu().numpy(), kt.grad.cpu().numpy(), ct.grad.cpu().numpy()
    # dL/dc is linear in c: compare with the exact adjoint sum 2 sum_i (g - y)_i J(k_i r_j)
    adj = 2.0 * orc.direct_sum(nu, k, r, g - y, np.arange(m))
    assert np.abs(gc - adj).max() <= 1e-8 * np.abs(adj).max()
    for j in rng.choice(m, 16, replace=False):
        fd = _fd_r(orc, nu, r, k, c, y, g, j, h)
        assert abs(gr[j] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(gr).max()), (j, gr[j], fd)
    for i in rng.choice(n, 16, replace=False):
        fd = _fd_k(orc, nu, r, k, c, y, g, i, h)
        assert abs(gk[i] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(gk).max()), (i, gk[i], fd)


def test_differentiation_full_size(cuda, orc):
    """nu = 1, N = M = 2e5 log-uniform r on [1e-3, 1e2] and k on [1e-2, 1e3], batch 8,
    y = H c0 + 1e-3 noise, loss ||H c0 - y||^2: forward against the exact sums, gradients wrt
    c, r, k (FP64, tol 1e-10) against central differences (step 1e-6) on 64 random
    coordinates.  The exact values of H c0 come from the direct FP64 evaluator (every pair
    summed on the GPU, no expansion); the differences themselves from the oracle."""
    import torch
    from nufht_b200 import _lib as L
    from nufht_b200.torch_ops import nufht
    rng = np.random.default_rng(2024)
    n = m = 200_000
    B, nu = 8, 1.0
    r = np.sort(10.0 ** rng.uniform(-3, 2, m))
    k = np.sort(10.0 ** rng.uniform(-2, 3, n))
    c0 = rng.standard_normal((m, B))
    rt = torch.tensor(r, device=cuda, requires_grad=True)
    kt = torch.tensor(k, device=cuda, requires_grad=True)
    ct = torch.tensor(c0, device=cuda, requires_grad=True)
    cf = np.asfortranarray(c0)
    gf = np.zeros((n, B), order="F")
    L.lib().add_dir_batch(L.dptr(gf), nu, L.dptr(r), L.dptr(cf), L.dptr(k), m, n, B, m, n)
    g = np.ascontiguousarray(gf)
    y = g + 1e-3 * rng.standard_normal((n, B))
    out = nufht(ct, rt, kt, nu, tol=1e-10)
    loss = ((out - torch.tensor(y, device=cuda)) ** 2).sum()
    loss.backward()
    gg = out.detach().cpu().numpy()
    # forward: within tol * ||c_t||_1 of the exact sums in every column
    assert (np.abs(gg - g).max(axis=0) / np.abs(c0).sum(axis=0)).max() <= 1e-10
    L0 = float(((g - y) ** 2).sum())
    assert abs(loss.item() - L0) <= 1e-6 * L0
    # The differences are taken around the computed forward value,
    # L(r_j +- h) = ||gg + (exact change of g) - y||^2, which checks the backward pass (the
    # transforms of orders 0 and 2 and the adjoint) on its own; the forward is checked above.
    gr, gk, gc = rt.grad.cpu().numpy(), kt.grad.cpu().numpy(), ct.grad.cpu().numpy()
    h = 1e-6
    bad = []
    for j in rng.choice(m, 22, replace=False):
        fd = _fd_r(orc, nu, r, k, c0, y, gg, j, h)
        if abs(gr[j] - fd) > 1e-5 * max(abs(fd), 1e-3 * np.abs(gr).max()):
            bad.append(("r", int(j), gr[j], fd))
    for i in rng.choice(n, 21, replace=False):
        fd = _fd_k(orc, nu, r, k, c0, y, gg, i, h)
        if abs(gk[i] - fd) > 1e-5 * max(abs(fd), 1e-3 * np.abs(gk).max()):
            bad.append(("k", int(i), gk[i], fd))
    for j, t in zip(rng.choice(m, 21, replace=False), rng.integers(0, B, 21)):
        # L is quadratic in c: the central difference is exact, 2 sum_i (g - y)[i,t] J(k_i r_j)
        fd = 2.0 * orc.direct_sum(nu, k, r[j:j + 1], (gg - y)[:, t], np.array([0]))[0, 0]
        if abs(gc[j, t] - fd) > 1e-5 * max(abs(fd), 1e-3 * np.abs(gc).max()):
            bad.append(("c", (int(j), int(t)), gc[j, t], fd))
    assert not bad, bad


def test_module_reuses_plans(cuda):
    import torch
    from nufht_b200.torch_ops import HankelTransform
    rng = np.random.default_rng(1)
    r = torch.tensor(np.sort(rng.uniform(0.1, 50, 2000)), device=cuda)
    k = torch.tensor(np.sort(rng.uniform(0.1, 40, 1500)), device=cuda)
    mod = HankelTransform(0.0)
    c = torch.randn(2000, 2, dtype=torch.float64, device=cuda, requires_grad=True)
    g1 = mod(c, r, k)
    plans = mod._plans
    g2 = mod(c, r, k)
    assert mod._plans is plans
    # the phases add into g with atomics from concurrent streams: equal up to summation order
    assert torch.allclose(g1, g2, rtol=0, atol=1e-13 * float(g1.abs().max()))
    g2.sum().backward()
    assert c.grad is not None and c.grad.shape == c.shape
