"""The allocation-free local-box entry point against the regular one.

nufht_b200_add_loc_batch_noalloc exists for callers that cannot allocate device memory at
call time (a fixed memory budget or pool, or allocation forbidden after start-up); it keeps
its scratch in a device array inside the library.  This file runs last (its name sorts
after the others) so that a run stopping at the first failure has run every other test;
it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _inputs(seed, m, n, B, z):
    rng = np.random.default_rng(seed)
    r = np.sort(rng.uniform(0.05, 3.0, m))
    k = np.sort(rng.uniform(0.01, 0.95 * z / 3.0, n))   # k r < z: the local regime
    c = rng.standard_normal((B, m))                      # column t = row t
    g0 = rng.standard_normal((B, n))
    return r, k, c, g0


@pytest.mark.parametrize("nu", [0.0, 3.0])
def test_noalloc_matches_add_loc_batch_twice(cuda, orc, nu):
    import torch
    from nufht_b200 import _lib as L
    lib = L.lib()
    rc, z, ka, K, coef = orc.plan_params(nu, 1e-8)
    assert rc == 0
    m, n, B = 5000, 3000, 6
    for call in range(2):  # two calls in a row: the shared scratch keeps the last call's contents
        r, k, c, g0 = _inputs(100 + call, m, n, B, z)
        d = lambda a: torch.tensor(a, dtype=torch.float64, device=cuda).contiguous()
        rd, kd, cd = d(r), d(k), d(c)
        g_ref = d(g0)
        lib.add_loc_batch(_ptr(g_ref), nu, _ptr(rd), _ptr(cd), _ptr(kd), m, n, K, B, m, n, None, None, None)
        g = d(g0)
        ret = lib.nufht_b200_add_loc_batch_noalloc(_ptr(g), nu, _ptr(rd), _ptr(cd), _ptr(kd), m, n, K, B, m, n,
                                                   None)
        torch.cuda.synchronize()
        assert ret == 0, L.strerror(ret)
        err = (g - g_ref).abs().max(dim=1).values.cpu().numpy() / np.abs(c).sum(axis=1)
        assert err.max() <= 1e-13, (call, err)          # same kernels: agreement to rounding
        assert not torch.equal(g, d(g0))                # something was added


def test_noalloc_rejects_oversized_call_without_touching_output(cuda):
    import torch
    from nufht_b200 import _lib as L
    lib = L.lib()
    m, n, B, K = 1_200_000, 128, 64, 14  # partial sums alone would need about 4.5 MB
    r = torch.linspace(0.01, 1.0, m, dtype=torch.float64, device=cuda)
    k = torch.linspace(0.01, 1.0, n, dtype=torch.float64, device=cuda)
    c = torch.zeros((B, m), dtype=torch.float64, device=cuda)
    g = torch.full((B, n), 7.0, dtype=torch.float64, device=cuda)
    ret = lib.nufht_b200_add_loc_batch_noalloc(_ptr(g), 0.0, _ptr(r), _ptr(c), _ptr(k), m, n, K, B, m, n, None)
    torch.cuda.synchronize()
    assert ret == L.NUFHT_E_TOO_LARGE
    assert bool((g == 7.0).all())


def test_noalloc_rejects_host_buffers_and_signs_negative_odd_orders(cuda, orc):
    """Buffers must be device memory of the current device (a host array is refused before
    any launch); a negative odd order adds the negated expansion (J_{-n} = (-1)^n J_n)."""
    import torch
    from nufht_b200 import _lib as L
    lib = L.lib()
    rc, z, ka, K, coef = orc.plan_params(3.0, 1e-8)
    m, n, B = 3000, 2000, 3
    r, k, c, g0 = _inputs(7, m, n, B, z)
    d = lambda a: torch.tensor(a, dtype=torch.float64, device=cuda).contiguous()
    rd, kd, cd = d(r), d(k), d(c)
    host_g = np.ascontiguousarray(g0)
    ret = lib.nufht_b200_add_loc_batch_noalloc(host_g.ctypes.data_as(ctypes.c_void_p), 3.0, _ptr(rd), _ptr(cd),
                                               _ptr(kd), m, n, K, B, m, n, None)
    assert ret == -400 and np.array_equal(host_g, g0)
    gp, gm = d(g0), d(g0)
    assert lib.nufht_b200_add_loc_batch_noalloc(_ptr(gp), 3.0, _ptr(rd), _ptr(cd), _ptr(kd), m, n, K, B, m, n,
                                                None) == 0
    torch.cuda.synchronize()
    assert lib.nufht_b200_add_loc_batch_noalloc(_ptr(gm), -3.0, _ptr(rd), _ptr(cd), _ptr(kd), m, n, K, B, m, n,
                                                None) == 0
    torch.cuda.synchronize()
    base = d(g0)
    err = ((gm - base) + (gp - base)).abs().max(dim=1).values.cpu().numpy() / np.abs(c).sum(axis=1)
    assert err.max() <= 1e-13
