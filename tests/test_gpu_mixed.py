"""Mixed precision (FP32 asymptotic boxes) against the oracle and the FP64 direct sum, with
the same bar as the FP64 path: max_i |g - g_ref| <= tol * ||c_t||_1 per column."""
import os

import numpy as np
import pytest

from conftest import col_err, grids

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nu,tol,kind,m,n,B,seed", [
    (0.0, 1e-8, "uniform", 4000, 3500, 8, 1),
    (0.0, 1e-6, "uniform", 3000, 4000, 3, 2),
    (1.0, 1e-8, "loguniform", 4000, 3000, 5, 3),
    (10.0, 1e-8, "uniform", 3000, 2500, 4, 4),
    (-3.0, 1e-8, "uniform", 2500, 2500, 2, 5),
    (0.5, 1e-8, "uniform", 2000, 2000, 3, 6),
])
def test_mixed_vs_oracle(cuda, orc, nu, tol, kind, m, n, B, seed):
    import torch
    from nufht_b200 import DevicePlan
    r, k = grids(kind, m, n, seed)
    if nu == 0.5:
        r, k = r + 1.0, k + 1.0  # half-integer method is judged away from the origin
    c = np.random.default_rng(seed).standard_normal((m, B))
    p = DevicePlan(nu, r, k, tol, mixed=True)
    assert p.info()["mixed"] == 1
    g = p(torch.tensor(c, device=cuda)).cpu().numpy()
    g_or = orc.nufht_batch(nu, r, k, c, tol)
    err = col_err(g, g_or, c)
    assert err.max() <= tol, err


def test_mixed_falls_back_to_fp64_below_1e9(cuda, orc):
    import torch
    from nufht_b200 import DevicePlan
    r, k = grids("uniform", 3000, 3000, 7)
    c = np.random.default_rng(7).standard_normal((3000, 2))
    p = DevicePlan(0.0, r, k, 1e-10, mixed=True)
    assert p.info()["mixed"] == 0
    g = p(torch.tensor(c, device=cuda)).cpu().numpy()
    assert col_err(g, orc.nufht_batch(0.0, r, k, c, 1e-10), c).max() <= 1e-10


def test_full_size_workload_both_precisions(cuda, orc):
    """N = M = 1e6 on (0, 1000], 4 columns: FP64 and mixed forms against the exact FP64
    sum at 96 sampled targets, and linearity in c."""
    import torch
    from nufht_b200 import DevicePlan
    N = 1_000_000
    rng = np.random.default_rng(1)
    r = np.sort(1000.0 * (1.0 - rng.random(N)))
    k = np.sort(1000.0 * (1.0 - rng.random(N)))
    c = np.random.default_rng(2).standard_normal((N, 4))
    idx = np.sort(np.random.default_rng(3).choice(N, 96, replace=False))
    exact = orc.direct_sum(0.0, r, k, c, idx)
    ct = torch.tensor(c, device=cuda)
    for mixed in (False, True):
        p = DevicePlan(0.0, r, k, 1e-8, mixed=mixed)
        g = p(ct)
        err = col_err(g.cpu().numpy()[idx], exact, c)
        assert err.max() <= 1e-8, (mixed, err)
        # linearity: H(2 c0 - c1) = 2 H c0 - H c1
        comb = p(2.0 * ct[:, 0] - ct[:, 1])
        lin = (comb - (2.0 * g[:, 0] - g[:, 1])).abs().max().item()
        assert lin <= 1e-8 * (2 * np.abs(c[:, 0]).sum() + np.abs(c[:, 1]).sum()), (mixed, lin)
        p.close()


def test_reference_entry_point_precision_switch(cuda, orc):
    """NUFHT_B200_PRECISION=mixed selects the mixed path for nufht_plan_init/nufht_batch."""
    from nufht_b200 import _pynufht as pn
    r, k = grids("uniform", 3000, 3000, 8)
    c = np.random.default_rng(8).standard_normal((3000, 3))
    os.environ["NUFHT_B200_PRECISION"] = "mixed"
    try:
        g = pn.nufht_batch(0.0, r, c, k, 1e-8)
    finally:
        del os.environ["NUFHT_B200_PRECISION"]
    assert col_err(g, orc.nufht_batch(0.0, r, k, c, 1e-8), c).max() <= 1e-8
