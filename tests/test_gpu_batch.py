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


def test_graph_batch_shared_plan_widths_and_pinning(cuda):
    """Items that share a plan at different widths, and a standalone run of a batched plan at a
    larger width: the batch keeps the buffers its graph recorded (pinned plan), so later
    launches still give the plan's results; destroying the batch releases the old buffers.
    The plan's handle may also be closed while the batch still uses it."""
    import torch
    from nufht_b200 import DevicePlan
    from nufht_b200.batch import TransformBatch
    rng = np.random.default_rng(6)
    r = np.sort(300.0 * (1.0 - rng.random(20000)))
    k = np.sort(200.0 * (1.0 - rng.random(15000)))
    p = DevicePlan(0.0, r, k, 1e-8)
    q = DevicePlan(1.0, k, r, 1e-8)
    ca = torch.tensor(rng.standard_normal((3, 20000)), device=cuda)
    cb = torch.tensor(rng.standard_normal((7, 20000)), device=cuda)
    cq = torch.tensor(rng.standard_normal((5, 15000)), device=cuda)
    ref = [p.execute_columns(ca).clone(), p.execute_columns(cb).clone(), q.execute_columns(cq).clone()]
    tb = TransformBatch([(p, ca), (p, cb), (q, cq)], branches=2)
    grid0, retired0, pins = p.buffers()
    assert pins == 1 and retired0 == 0
    out = [o.clone() for o in tb.launch()]
    torch.cuda.synchronize()
    for a, b in zip(out, ref):
        assert torch.allclose(a, b, rtol=0, atol=1e-12 * float(b.abs().max()))
    # the plan alone at a larger width: new workspace, the graph's one kept
    wide = torch.tensor(rng.standard_normal((24, 20000)), device=cuda)
    wide_out = p.execute_columns(wide).clone()
    grid1, retired1, _ = p.buffers()
    assert grid1 != grid0 and retired1 >= 1
    q.close()  # the batch still holds the plan
    for o in tb.outputs:
        o.fill_(np.nan)
    out2 = tb.launch()
    torch.cuda.synchronize()
    for a, b in zip(out2, ref):
        assert torch.allclose(a, b, rtol=0, atol=1e-12 * float(b.abs().max()))
    tb.close()
    _, retired2, pins2 = p.buffers()
    assert pins2 == 0 and retired2 == 0
    assert torch.allclose(p.execute_columns(wide), wide_out, rtol=0, atol=1e-12 * float(wide_out.abs().max()))
    p.close()
