"""The stress workload: nu = 100, N = M = 4e6, |r| from a mixture of three Gaussians (means
200, 800, 1500; sd 50) clipped to (0, 2000], k uniform on (0, 2000], batch 64, tol 1e-8;
forward in mixed precision (mixed="averaged": FP32 asymptotic boxes, checked on the N(0,1)
columns of the workload) and the autograd backward with respect to c (the adjoint
transform, planned and run afresh: nothing of the forward is stored but c), on one GPU.  The reference's
tables leave K_asy = 10 empty at this order (its asymptotic boxes would get z_split = 0), so
the plans use the extended tables, and the results are checked against the oracle's direct
sums only."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _grids(rng, n):
    means = np.array([200.0, 800.0, 1500.0])
    r = rng.normal(means[rng.integers(0, 3, n)], 50.0)
    r = np.clip(np.abs(r), 1e-9, 2000.0)
    k = 2000.0 * (1.0 - rng.random(n))
    return np.sort(r), np.sort(k)


def test_stress_nu100_forward_and_backward(cuda, orc):
    import torch
    from nufht_b200.torch_ops import HankelTransform
    rng = np.random.default_rng(100)
    n = 4_000_000
    B, nu, tol = 64, 100.0, 1e-8
    r, k = _grids(rng, n)
    rt = torch.tensor(r, device=cuda)
    kt = torch.tensor(k, device=cuda)
    c = torch.randn((n, B), dtype=torch.float64, device=cuda, generator=torch.Generator(device=cuda).manual_seed(3))
    c.requires_grad_(True)
    mod = HankelTransform(nu, tol=tol, mixed="averaged", extended_tables=True)
    g = mod(c, rt, kt)
    assert mod._plans.plan(nu, False).info()["mixed"] == 1
    u = torch.randn((n, B), dtype=torch.float64, device=cuda, generator=torch.Generator(device=cuda).manual_seed(4))
    (g * u).sum().backward()
    dc = c.grad
    ch = c.detach().cpu().numpy()
    uh = u.cpu().numpy()
    idx = np.sort(rng.choice(n, 12, replace=False))
    ex = orc.direct_sum(nu, r, k, ch, idx)
    fwd = np.abs(g.detach()[idx].cpu().numpy() - ex).max(axis=0) / np.abs(ch).sum(axis=0)
    assert fwd.max() <= tol, fwd.max()
    jdx = np.sort(rng.choice(n, 12, replace=False))
    exb = orc.direct_sum(nu, k, r, uh, jdx)
    bwd = np.abs(dc[jdx].cpu().numpy() - exb).max(axis=0) / np.abs(uh).sum(axis=0)
    assert bwd.max() <= tol, bwd.max()
    mod.release()
