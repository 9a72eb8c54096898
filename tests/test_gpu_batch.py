"""Many independent transforms in one CUDA-graph launch: 256 problems drawn like the
batching workload (nu in {0, 1/2, 1, 2, 7/2, 10}, N and M log-uniform in [1e3, 1e5], r and k
uniform on (0, R] and (0, K] with R, K log-uniform in [10, 1e3], 1-16 columns, tol in
{1e-4, 1e-8, 1e-12}), checked against the oracle's direct sums at sampled targets and
against the same plans executed one by one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems(rng, count, nmax=100_000):
    out = []
    for _ in range(count):
        nu = float(rng.choice([0.0, 0.5, 1.0, 2.0, 3.5, 10.0]))
        N = int(10.0 ** rng.uniform(3, np.log10(nmax)))
        M = int(10.0 ** rng.uniform(3, np.log10(nmax)))
        R = 10.0 ** rng.uniform(1, 3)
        K = 10.0 ** rng.uniform(1, 3)
        r = np.sort(R * (1.0 - rng.random(N)))
        k = np.sort(K * (1.0 - rng.random(M)))
        B = int(rng.integers(1, 17))
        tol = float(rng.choice([1e-4, 1e-8, 1e-12]))
        c = rng.standard_normal((B, N))
        out.append((nu, r, k, B, tol, c))
    return out


def test_graph_batch_matches_oracle_and_single_runs(cuda, orc):
    import torch
    from nufht_b200 import DevicePlan
    from nufht_b200.batch import TransformBatch
    rng = np.random.default_rng(4)
    probs = _problems(rng, 256)
    plans, items = [], []
    for nu, r, k, B, tol, c in probs:
        p = DevicePlan(nu, r, k, tol)
        plans.append(p)
        items.append((p, torch.tensor(c, device=cuda)))
    tb = TransformBatch(items)
    info = tb.info()
    assert info["branches"] >= 1 and info["kernel_nodes"] >= len(probs)
    for o in tb.outputs:
        o.fill_(np.nan)
    tb.launch()
    torch.cuda.synchronize()
    outs = [o.cpu().numpy() for o in tb.outputs]
    worst = 0.0
    for q, ((nu, r, k, B, tol, c), (p, ct)) in enumerate(zip(probs, items)):
        g = outs[q]
        assert np.isfinite(g).all(), q
        # the same plan run alone gives the same values (up to summation order)
        single = p.execute_columns(ct).cpu().numpy()
        l1 = np.abs(c).sum(axis=1)
        assert (np.abs(single - g).max(axis=1) / l1).max() <= 1e-13, q
        idx = np.unique(rng.integers(0, len(k), 6))
        ex = orc.direct_sum(nu, r, k, c.T, idx).T  # (B, len(idx))
        err = (np.abs(g[:, idx] - ex).max(axis=1) / l1).max()
        worst = max(worst, err / tol)
        assert err <= tol, (q, nu, len(r), len(k), B, tol, err)
    tb.close()
    for p in plans:
        p.close()


def test_graph_batch_fixed_branches_and_relaunch(cuda):
    import torch
    from nufht_b200 import DevicePlan
    from nufht_b200.batch import TransformBatch
    rng = np.random.default_rng(5)
    probs = _problems(rng, 12, nmax=20_000)
    items = [(DevicePlan(nu, r, k, tol), torch.tensor(c, device=cuda)) for nu, r, k, B, tol, c in probs]
    tb = TransformBatch(items, branches=3)
    assert tb.info()["branches"] == 3
    first = [o.clone() for o in tb.launch()]
    for _, c in items:
        c.mul_(2.0)  # inputs are read at every launch
    second = tb.launch()
    torch.cuda.synchronize()
    for a, b in zip(first, second):
        assert torch.allclose(b, 2.0 * a, rtol=0, atol=1e-12 * float(a.abs().max()) + 1e-300)
    tb.close()
