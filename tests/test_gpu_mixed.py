"""Mixed precision against the oracle and the FP64 direct sum, with the same bar as the FP64
path, max_i |g - g_ref| <= tol * ||c_t||_1 per column: mixed=True (FP32 asymptotic boxes
where the planner's worst-case FP32 error model allows it, FP64 elsewhere) on any columns,
mixed="averaged" (FP32 regardless) on columns of N(0,1) entries, and the averaged form's
single-source worst case against the model's bound."""
import os

import numpy as np
import pytest

from conftest import col_err, grids

pytestmark = pytest.mark.gpu


def _stats(p):
    return p.stats()


@pytest.mark.parametrize("nu,tol,kind,m,n,B,seed,fp32", [
    (0.0, 1e-5, "uniform", 4000, 3500, 8, 1, True),
    (0.0, 1e-8, "uniform", 4000, 3500, 8, 1, False),
    (1.0, 1e-5, "loguniform", 4000, 3000, 5, 3, True),
    (10.0, 1e-4, "uniform", 3000, 2500, 4, 4, True),
    (-3.0, 1e-5, "uniform", 2500, 2500, 2, 5, True),
    (0.5, 1e-5, "uniform", 2000, 2000, 3, 6, True),
    (0.0, 1e-6, "uniform", 3000, 4000, 3, 2, None),
])
def test_mixed_vs_oracle(cuda, orc, nu, tol, kind, m, n, B, seed, fp32):
    import torch
    from nufht_b200 import DevicePlan
    r, k = grids(kind, m, n, seed)
    if nu == 0.5:
        r, k = r + 1.0, k + 1.0  # half-integer method is checked away from the origin
    c = np.random.default_rng(seed).standard_normal((m, B))
    p = DevicePlan(nu, r, k, tol, mixed=True)
    st = _stats(p)
    # FP32 exactly where the modelled worst case is within tol / 4
    assert p.info()["mixed"] == int(st[14] <= 0.25 * tol) == st[13], (st[13], st[14])
    if fp32 is not None:
        assert p.info()["mixed"] == int(fp32), st[14]
    g = p(torch.tensor(c, device=cuda)).cpu().numpy()
    g_or = orc.nufht_batch(nu, r, k, c, tol)
    err = col_err(g, g_or, c)
    assert err.max() <= tol, err
    p.close()


@pytest.mark.parametrize("nu,tol,kind,m,n,B,seed", [
    (0.0, 1e-8, "uniform", 4000, 3500, 8, 1),
    (1.0, 1e-8, "loguniform", 4000, 3000, 5, 3),
    (10.0, 1e-8, "uniform", 3000, 2500, 4, 4),
    (-3.0, 1e-8, "uniform", 2500, 2500, 2, 5),
    (0.5, 1e-8, "uniform", 2000, 2000, 3, 6),
])
def test_mixed_averaged_vs_oracle(cuda, orc, nu, tol, kind, m, n, B, seed):
    import torch
    from nufht_b200 import DevicePlan
    r, k = grids(kind, m, n, seed)
    if nu == 0.5:
        r, k = r + 1.0, k + 1.0
    c = np.random.default_rng(seed).standard_normal((m, B))
    p = DevicePlan(nu, r, k, tol, mixed="averaged")
    assert p.info()["mixed"] == 1
    g = p(torch.tensor(c, device=cuda)).cpu().numpy()
    err = col_err(g, orc.nufht_batch(nu, r, k, c, tol), c)
    assert err.max() <= tol, err
    p.close()


@pytest.mark.parametrize("tol,fp32", [(1e-5, True), (1e-8, False)])
def test_mixed_single_sources(cuda, orc, tol, fp32):
    """Columns with all their mass on one source (no averaging of FP32 rounding over many
    sources): one far source, one mid-range source, and a random column dominated by a
    spike 1e3 times its entries, against the exact FP64 sums.  At tol 1e-8 FP32 rounding of
    a single source (about 3e-7 of its weight) would exceed the tolerance, so the plan keeps
    FP64."""
    import torch
    from nufht_b200 import DevicePlan
    r, k = grids("uniform", 4000, 3500, 11)
    c = np.zeros((4000, 3))
    c[3900, 0] = 1.0
    c[2000, 1] = -1.0
    c[:, 2] = np.random.default_rng(11).standard_normal(4000)
    c[3500, 2] = 1e3
    p = DevicePlan(0.0, r, k, tol, mixed=True)
    assert p.info()["mixed"] == int(fp32)
    g = p(torch.tensor(c, device=cuda)).cpu().numpy()
    exact = orc.direct_sum(0.0, r, k, c, np.arange(3500))
    err = col_err(g, exact, c)
    assert err.max() <= tol, err
    p.close()
    # The averaged form keeps FP32 at 1e-8: the single-source columns stay within the
    # planner's worst-case bound (which is above the tolerance there).
    q = DevicePlan(0.0, r, k, tol, mixed="averaged")
    bound = q.stats()[14]
    assert q.info()["mixed"] == 1
    ga = q(torch.tensor(c, device=cuda)).cpu().numpy()
    assert col_err(ga, exact, c).max() <= tol + bound, (col_err(ga, exact, c), bound)
    q.close()


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
    sum at 96 sampled targets (exact at tol 1e-8, so within tol 1e-5 as well), and
    linearity in c."""
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
    # mixed at 1e-8 keeps FP64 (FP32 rounding could exceed the tolerance); at 1e-5 it is FP32
    for mixed, tol, fp32 in ((False, 1e-8, 0), (True, 1e-8, 0), (True, 1e-5, 1), ("averaged", 1e-8, 1)):
        p = DevicePlan(0.0, r, k, tol, mixed=mixed)
        assert p.info()["mixed"] == fp32
        g = p(ct)
        err = col_err(g.cpu().numpy()[idx], exact, c)
        assert err.max() <= tol, (mixed, tol, err)
        # linearity: H(2 c0 - c1) = 2 H c0 - H c1
        comb = p(2.0 * ct[:, 0] - ct[:, 1])
        lin = (comb - (2.0 * g[:, 0] - g[:, 1])).abs().max().item()
        assert lin <= tol * (2 * np.abs(c[:, 0]).sum() + np.abs(c[:, 1]).sum()), (mixed, tol, lin)
        p.close()


def test_reference_entry_point_precision_switch(cuda, orc):
    """NUFHT_B200_PRECISION=mixed / mixed-averaged select the mixed paths for
    nufht_plan_init / nufht_batch."""
    from nufht_b200 import _pynufht as pn
    r, k = grids("uniform", 3000, 3000, 8)
    c = np.random.default_rng(8).standard_normal((3000, 3))
    for pr, tol in (("mixed", 1e-5), ("mixed-averaged", 1e-8)):
        os.environ["NUFHT_B200_PRECISION"] = pr
        try:
            g = pn.nufht_batch(0.0, r, c, k, tol)
        finally:
            del os.environ["NUFHT_B200_PRECISION"]
        assert col_err(g, orc.nufht_batch(0.0, r, k, c, tol), c).max() <= tol


@pytest.fixture(scope="module")
def cfg2_exact(orc):
    """The 1e6-point workload (N = M = 1e6 on (0, 1000], batch 32 of N(0,1)) and the oracle's
    exact FP64 direct sums (every source, Kahan-compensated, on all host cores) at 2000
    sampled targets."""
    N, B = 1_000_000, 32
    rng = np.random.default_rng(1)
    r = np.sort(1000.0 * (1.0 - rng.random(N)))
    k = np.sort(1000.0 * (1.0 - rng.random(N)))
    c = np.random.default_rng(2).standard_normal((N, B))
    idx = np.sort(np.random.default_rng(3).choice(N, 2000, replace=False))
    ex = orc.direct_sum(0.0, r, k, c, idx)
    return r, k, c, idx, ex


@pytest.mark.parametrize("tol", [1e-6, 1e-8, 1e-10])
def test_cfg2_full_size_tolerances(cuda, cfg2_exact, tol):
    """N = M = 1e6 on (0, 1000], batch 32 of N(0,1), tol 1e-6, 1e-8 and 1e-10: the plain FP64
    form and both mixed forms against the oracle's FP64 direct sums at 2000 sampled targets
    (32 columns), and the library's own GPU direct evaluator as a second cross-check."""
    import torch
    from nufht_b200 import DevicePlan
    from nufht_b200 import _lib as L
    r, k, c, idx, ex = cfg2_exact
    N, B = c.shape
    ks = np.ascontiguousarray(k[idx])
    gd = np.zeros((len(idx), B), order="F")
    cf = np.asfortranarray(c)
    L.lib().add_dir_batch(L.dptr(gd), 0.0, L.dptr(r), L.dptr(cf), L.dptr(ks), N, len(idx), B, N, len(idx))
    assert col_err(gd, ex, c).max() <= 1e-12
    ct = torch.tensor(c, device=cuda)
    it = torch.tensor(idx, device=cuda)
    for mixed in (False, True, "averaged"):
        p = DevicePlan(0.0, r, k, tol, mixed=mixed)
        # FP32 only where allowed: never below 1e-9; strict mode only within its bound
        expect = int(tol >= 1e-9 and (mixed == "averaged" or (mixed is True and p.stats()[14] <= 0.25 * tol)))
        assert p.info()["mixed"] == expect
        g = p(ct)[it].cpu().numpy()
        err = col_err(g, ex, c)
        assert err.max() <= tol, (mixed, tol, err.max())
        p.close()
