"""GPU parity: the CUDA path (through the C ABI) against the oracle, the reference's golden
outputs and known answers.  Bar: max_i |g_gpu - g_ref| <= tol * ||c_t||_1 per column t."""
import ctypes
import math
import os

import numpy as np
import pytest

from conftest import col_err, grids

pytestmark = pytest.mark.gpu


def test_device_bessel_vs_mpmath(cuda, golden):
    import torch
    from nufht_b200 import _lib as L
    g = golden("bessel_golden.npz")
    # absolute error bound 1e-14 (the transform's accuracy is measured relative to ||c||_1)
    for nu in np.unique(g["nu"]):
        sel = g["nu"] == nu
        x = torch.tensor(g["x"][sel], dtype=torch.float64, device=cuda)
        out = torch.empty_like(x)
        rc = L.lib().nufht_b200_besselj(float(nu), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                        x.numel(), None)
        assert rc == 0
        torch.cuda.synchronize()
        err = np.abs(out.cpu().numpy() - g["j"][sel])
        assert err.max() < 1e-14, (nu, err.max(), g["x"][sel][err.argmax()])


def test_golden_reference_outputs(cuda, golden):
    """Outputs of the reference's own driver (oracle/_ref, exact type-3 sums) reproduced by
    the drop-in _pynufht.nufht_batch on the GPU."""
    from nufht_b200 import _pynufht as pn
    e = golden("e2e_golden.npz")
    for name in e["names"]:
        nu, tol, B = e[name + "_meta"]
        r, k, c = e[name + "_r"], e[name + "_k"], e[name + "_c"]
        g = pn.nufht_batch(nu, r, c, k, tol)
        assert g.shape == (len(k), int(B)) and g.flags["C_CONTIGUOUS"]
        err = col_err(g, e[name + "_g"], c)
        assert err.max() <= tol, (name, err)


def test_cfg1_gauss_legendre(cuda, orc):
    """nu=0; r = 10000 Gauss-Legendre nodes on [0,50]; c = r w x, x ~ N(0,1) (seed 0), 4
    columns; k = 200 points 10(i+1)/200; tol 1e-8."""
    from nufht_b200 import _pynufht as pn
    x, w = np.polynomial.legendre.leggauss(10000)
    r, w = 25 * (x + 1), 25 * w
    c = (r * w)[:, None] * np.random.default_rng(0).standard_normal((10000, 4))
    k = 10 * np.arange(1, 201) / 200
    g = pn.nufht_batch(0.0, r, c, k, 1e-8)
    g_or = orc.nufht_batch(0.0, r, k, c, 1e-8)
    assert col_err(g, g_or, c).max() <= 1e-8
    idx = np.arange(200)
    gd = orc.direct_sum(0.0, r, k, c, idx)
    assert col_err(g, gd, c).max() <= 1e-8


def test_known_answer_gaussian(cuda):
    """python/run_pynufht_test.py through the drop-in pn.nufht: |g - exp(-k^2/2)| ~ 1e-13
    (notebooks/nufht_batch_example.ipynb:190 records 9.96e-14)."""
    from nufht_b200 import _pynufht as pn
    x, w = np.polynomial.legendre.leggauss(1000)
    r, w = 5 * (x + 1), 5 * w
    cs = r * np.exp(-0.5 * r * r) * w
    k = 10 * np.arange(1, 101) / 100
    g = pn.nufht(0.0, r, cs, k)
    assert np.abs(g - np.exp(-0.5 * k * k)).max() < 2e-13
    gb = pn.nufht_batch(0.0, r, np.stack([cs, 0.5 * cs], 1), k)
    assert np.abs(gb[:, 1] - 0.5 * np.exp(-0.5 * k * k)).max() < 1e-13
    gl = pn.nufht_batch_loop(0.0, r, np.stack([cs, 0.5 * cs], 1), k)
    assert np.abs(gl - gb).max() < 1e-13


def test_known_answer_half_integer(cuda, orc):
    """src/test_nufht.c (nu = 1/2, two columns) against the oracle's same-method result."""
    from nufht_b200 import _pynufht as pn
    x, w = np.polynomial.legendre.leggauss(10000)
    r, w = 5 * (x + 1), 5 * w
    cs = np.stack([r ** 1.5 * (1 + r * r) ** -n * w for n in (2, 3)], 1)
    k = 10 * np.arange(1, 101) / 100
    g = pn.nufht_batch(0.5, r, cs, k)
    g_or = orc.nufht_batch(0.5, r, k, cs, 1e-8)
    assert col_err(g, g_or, cs).max() <= 1e-8
    num = np.sqrt(np.pi / (2 * k))[:, None] * g
    an = np.stack([np.pi / 4 * np.exp(-k), np.pi / 16 * (1 + k) * np.exp(-k)], 1)
    tail = np.stack([10.0 ** (2 - 2 * n) / (2 * n - 2) / k for n in (2, 3)], 1)
    assert np.all(np.abs(num - an) <= tail + 1e-8)


CASES = [  # nu, tol, kind, m, n, B, seed
    (0.0, 1e-6, "uniform", 4000, 3500, 5, 1),
    (0.0, 1e-10, "uniform", 3000, 4000, 3, 2),
    (0.0, 1e-12, "loguniform", 3000, 3000, 2, 3),
    (1.0, 1e-8, "loguniform", 4000, 3000, 8, 4),
    (2.0, 1e-8, "uniform", 3000, 3000, 1, 5),
    (3.0, 1e-4, "uniform", 2500, 3000, 17, 6),
    (10.0, 1e-8, "uniform", 3000, 2500, 4, 7),
    (10.0, 1e-12, "uniform", 2000, 2000, 2, 8),
    (-1.0, 1e-8, "uniform", 3000, 3000, 1, 9),
    (-3.0, 1e-8, "uniform", 3000, 3000, 3, 10),
    (34.0, 1e-8, "uniform", 2000, 2000, 2, 11),
    (0.0, 1e-8, "uniform", 3000, 3000, 40, 12),
]


@pytest.mark.parametrize("nu,tol,kind,m,n,B,seed", CASES)
def test_random_vs_oracle(cuda, orc, nu, tol, kind, m, n, B, seed):
    from nufht_b200 import _pynufht as pn
    r, k = grids(kind, m, n, seed)
    c = np.random.default_rng(seed).standard_normal((m, B))
    g = pn.nufht_batch(nu, r, c, k, tol)
    g_or = orc.nufht_batch(nu, r, k, c, tol)
    err = col_err(g, g_or, c)
    assert err.max() <= tol, err


@pytest.mark.parametrize("nu", [1.5, 3.5])
def test_half_integer_away_from_origin(cuda, orc, nu):
    """Half-integer orders use the terminating Hankel expansion over the whole rectangle
    (src/fast_hankel_nufht.c:1052-1078); with k r >= 1 both sides agree to tol."""
    from nufht_b200 import _pynufht as pn
    rng = np.random.default_rng(3)
    r = np.sort(rng.uniform(1, 60, 2000))
    k = np.sort(rng.uniform(1, 40, 1500))
    c = rng.standard_normal((2000, 3))
    g = pn.nufht_batch(nu, r, c, k, 1e-8)
    g_or = orc.nufht_batch(nu, r, k, c, 1e-8)
    assert col_err(g, g_or, c).max() <= 1e-8
    gd = orc.direct_sum(nu, r, k, c, np.arange(0, 1500, 11))
    assert col_err(g[::11], gd, c).max() <= 1e-8


def test_leading_dimensions_and_device_pointers(cuda, orc):
    import torch
    from nufht_b200 import _lib as L
    lib = L.lib()
    r, k = grids("uniform", 3000, 2000, 21)
    m, n, B = 3000, 2000, 3
    c = np.random.default_rng(2).standard_normal((m, B))
    ldc, ldg = m + 7, n + 5
    cbuf = np.full((ldc, B), 123.0, order="F")
    cbuf[:m] = c
    gbuf = np.full((ldg, B), 77.0, order="F")
    plan = L.NufhtPlan()
    assert lib.nufht_plan_init(ctypes.byref(plan), 0.0, L.dptr(r), m, L.dptr(k), n, None) == 0
    assert lib.nufht_batch(ctypes.byref(plan), L.dptr(cbuf), ldc, L.dptr(gbuf), ldg, B, None) == 0
    g_or = orc.nufht_batch(0.0, r, k, c, 1e-8)
    assert col_err(gbuf[:n], g_or, c).max() <= 1e-8
    assert np.all(gbuf[n:] == 77.0)  # rows beyond n untouched
    # device pointers through the same reference entry point
    cd = torch.tensor(cbuf.T.copy(), device=cuda)  # (B, ldc) contiguous = column-major ldc
    gd = torch.zeros((B, ldg), dtype=torch.float64, device=cuda)
    assert lib.nufht_batch(ctypes.byref(plan), ctypes.c_void_p(cd.data_ptr()), ldc,
                           ctypes.c_void_p(gd.data_ptr()), ldg, B, None) == 0
    torch.cuda.synchronize()
    assert np.abs(gd.cpu().numpy().T[:n] - gbuf[:n]).max() < 1e-12
    lib.nufht_plan_free(ctypes.byref(plan))


def test_batch_layouts(cuda, orc):
    """nufht_b200_batch_layout: every combination of row-major (C-order) and column-major cs
    and gs, with padded leading dimensions, host and device pointers, against the oracle;
    _pynufht.nufht_batch on C-order, Fortran-order and strided cs gives a C-order result."""
    import torch
    from nufht_b200 import _lib as L
    from nufht_b200 import _pynufht as pn
    lib = L.lib()
    r, k = grids("uniform", 3000, 2000, 22)
    m, n, B = 3000, 2000, 5
    c = np.random.default_rng(3).standard_normal((m, B))
    g_or = orc.nufht_batch(0.0, r, k, c, 1e-8)
    plan = L.NufhtPlan()
    assert lib.nufht_plan_init(ctypes.byref(plan), 0.0, L.dptr(r), m, L.dptr(k), n, None) == 0
    for c_row in (0, 1):
        for g_row in (0, 1):
            ldc = (B + 3) if c_row else (m + 7)
            ldg = (B + 2) if g_row else (n + 5)
            cbuf = np.full((m, ldc) if c_row else (ldc, B), 123.0, order="C" if c_row else "F")
            cbuf[:m, :B] = c
            gbuf = np.full((n, ldg) if g_row else (ldg, B), 77.0, order="C" if g_row else "F")
            assert lib.nufht_b200_batch_layout(ctypes.byref(plan), L.dptr(cbuf), c_row, ldc, L.dptr(gbuf), g_row,
                                               ldg, B) == 0
            assert col_err(gbuf[:n, :B], g_or, c).max() <= 1e-8, (c_row, g_row)
            assert np.all(gbuf[n:] == 77.0) and np.all(gbuf[:, B:] == 77.0)  # padding untouched
            # device pointers
            cd = torch.tensor(np.ascontiguousarray(cbuf if c_row else cbuf.T), device=cuda)
            gd = torch.full((n, ldg) if g_row else (B, ldg), 77.0, dtype=torch.float64, device=cuda)
            assert lib.nufht_b200_batch_layout(ctypes.byref(plan), ctypes.c_void_p(cd.data_ptr()), c_row, ldc,
                                               ctypes.c_void_p(gd.data_ptr()), g_row, ldg, B) == 0
            torch.cuda.synchronize()
            gh = gd.cpu().numpy()
            gh = gh[:n, :B] if g_row else gh.T[:n, :B]
            assert np.abs(gh - gbuf[:n, :B]).max() <= 1e-12 * np.abs(c).sum(axis=0).max()
    assert lib.nufht_b200_batch_layout(ctypes.byref(plan), L.dptr(c), 2, B, L.dptr(g_or), 1, B, B) == -400
    assert lib.nufht_b200_batch_layout(ctypes.byref(plan), L.dptr(c), 1, B - 1, L.dptr(g_or), 1, B, B) == -401
    lib.nufht_plan_free(ctypes.byref(plan))
    for cs in (np.ascontiguousarray(c), np.asfortranarray(c), np.ascontiguousarray(np.repeat(c, 2, axis=1))[:, ::2]):
        g = pn.nufht_batch(0.0, r, cs, k, 1e-8)
        assert g.flags.c_contiguous and g.shape == (n, B)
        assert col_err(g, g_or, c).max() <= 1e-8


def test_device_plan_torch(cuda, orc):
    import torch
    from nufht_b200 import DevicePlan
    r, k = grids("loguniform", 5000, 4000, 22)
    c = np.random.default_rng(3).standard_normal((5000, 6))
    p = DevicePlan(1.0, r, k, 1e-8)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        g = p(torch.tensor(c, device=cuda))
    s.synchronize()
    g_or = orc.nufht_batch(1.0, r, k, c, 1e-8)
    assert col_err(g.cpu().numpy(), g_or, c).max() <= 1e-8
    info = p.info()
    assert info["n_asy"] > 0 and info["workspace_bytes"] > 0
    g1 = p(torch.tensor(c[:, 0], device=cuda))
    assert g1.shape == (4000,)
    assert torch.allclose(g1, g[:, 0], atol=1e-12, rtol=0)


@pytest.mark.parametrize("shape", ["m1", "n1", "all_loc", "all_asy", "ties", "tiny"])
def test_edge_cases(cuda, orc, shape):
    from nufht_b200 import _pynufht as pn
    rng = np.random.default_rng(4)
    if shape == "m1":
        r, k = np.array([3.7]), np.sort(rng.uniform(0.01, 50, 20000))
    elif shape == "n1":
        r, k = np.sort(rng.uniform(0.01, 50, 20000)), np.array([2.2])
    elif shape == "all_loc":
        r, k = np.sort(rng.uniform(0.0, 2, 3000)), np.sort(rng.uniform(0.0, 2, 3000))
    elif shape == "all_asy":
        r, k = np.sort(rng.uniform(20, 40, 3000)), np.sort(rng.uniform(20, 40, 3000))
    elif shape == "ties":
        r = np.sort(np.round(rng.uniform(0.1, 30, 4000), 0))
        k = np.sort(np.round(rng.uniform(0.1, 30, 3000), 1))
    else:
        r, k = np.array([0.5, 1.0, 2.0]), np.array([0.0, 1.0])
    c = rng.standard_normal((len(r), 2))
    g = pn.nufht_batch(0.0, r, c, k)
    g_or = orc.nufht_batch(0.0, r, k, c, 1e-8)
    assert col_err(g, g_or, c).max() <= 1e-8


def test_negative_odd_order_sign_batch1(cuda, orc):
    """Deliberate deviation: J_{-1} = -J_1 for every batch size (the reference negates
    twice when batch == 1)."""
    from nufht_b200 import _pynufht as pn
    r, k = grids("uniform", 2000, 2000, 30)
    c = np.random.default_rng(5).standard_normal(2000)
    g_neg = pn.nufht(-1.0, r, c, k)
    g_pos = pn.nufht(1.0, r, c, k)
    assert np.abs(g_neg + g_pos).max() < 1e-13 * np.abs(c).sum()
    g_or = orc.nufht_batch(-1.0, r, k, c[:, None], 1e-8, faithful=False)[:, 0]
    assert np.abs(g_neg - g_or).max() <= 1e-8 * np.abs(c).sum()


@pytest.mark.parametrize("kind", ["dir", "loc", "asy"])
def test_single_box_evaluators(cuda, orc, kind):
    """add_dir_batch / add_loc_batch / add_asy_batch add one box's contribution to gs."""
    from nufht_b200 import _lib as L
    lib = L.lib()
    rng = np.random.default_rng(6)
    rc, z, ka, kl, coef = orc.plan_params(2.0, 1e-8)
    if kind == "asy":
        r, k = np.sort(rng.uniform(5, 30, 1500)), np.sort(rng.uniform(z / 5 + 0.1, 12, 1200))
    elif kind == "loc":
        r, k = np.sort(rng.uniform(0.1, 3, 1500)), np.sort(rng.uniform(0.01, z / 3 - 0.1, 1200))
    else:
        r, k = np.sort(rng.uniform(0.1, 10, 300)), np.sort(rng.uniform(0.1, 10, 200))
    m, n, B = len(r), len(k), 3
    c = np.asfortranarray(rng.standard_normal((m, B)))
    g0 = np.asfortranarray(rng.standard_normal((n, B)))
    g = g0.copy(order="F")
    if kind == "dir":
        lib.add_dir_batch(L.dptr(g), 2.0, L.dptr(r), L.dptr(c), L.dptr(k), m, n, B, m, n)
    elif kind == "loc":
        lib.add_loc_batch(L.dptr(g), 2.0, L.dptr(r), L.dptr(c), L.dptr(k), m, n, kl, B, m, n, None, None, None)
    else:
        cf = np.ascontiguousarray(coef)
        lib.add_asy_batch(L.dptr(g), 2.0, L.dptr(r), L.dptr(c), L.dptr(k), m, n, ka, 1e-8, L.dptr(cf), B, m, n,
                          None, None)
    gd = orc.direct_sum(2.0, r, k, c, np.arange(n))
    assert col_err(g - g0, gd, c).max() <= 1e-8


@pytest.mark.parametrize("nu", [0.0, 1.0, 10.0, 100.0])
@pytest.mark.parametrize("shape", ["thin", "tall"])
def test_direct_box_large_against_oracle(cuda, orc, nu, shape):
    """add_dir_batch (the direct-box kernel) on large boxes whose k r runs through the
    transition region of J_nu (0 < k r <= 300): thin (48 targets x 1e5 sources, several
    threads per target) and tall (3000 targets x 400 sources), against the oracle's FP64
    direct sums at every target.  Bar: 1e-12 ||c_t||_1 per column."""
    from nufht_b200 import _lib as L
    lib = L.lib()
    rng = np.random.default_rng(int(nu) + (0 if shape == "thin" else 1000))
    if shape == "thin":
        m, n = 100_000, 48
    else:
        m, n = 400, 3000
    r = np.sort(300.0 * (1.0 - rng.random(m)))
    k = np.sort(0.05 + 0.95 * rng.random(n))
    B = 5
    c = np.asfortranarray(rng.standard_normal((m, B)))
    g = np.zeros((n, B), order="F")
    lib.add_dir_batch(L.dptr(g), nu, L.dptr(r), L.dptr(c), L.dptr(k), m, n, B, m, n)
    gd = orc.direct_sum(nu, r, k, c, np.arange(n))
    assert col_err(g, gd, c).max() <= 1e-12, (nu, shape)


@pytest.mark.parametrize("nu,B,K,ni", [(0.0, 1, None, 1200), (3.0, 70, None, 333), (10.0, 5, None, 129),
                                        (100.0, 9, 200, 300), (-7.0, 33, None, 17)])
def test_local_box_tensor_core_contractions(cuda, orc, nu, B, K, ni):
    """add_loc_batch on the FP64 tensor-core kernels (Chebyshev projection and Bessel-product
    evaluation as DMMA tiles): Wimp degrees from the tables and a degree of 200 at order 100
    (Bessel tables of 251 orders per target), one column, more than one 64-column pass, target
    counts that are not multiples of the tile, against the oracle's direct sums."""
    from nufht_b200 import _lib as L
    lib = L.lib()
    rng = np.random.default_rng(int(abs(nu)) + B)
    rc, z, ka, kl, coef = orc.plan_params(abs(nu), 1e-8)
    if K is None:
        K = kl
        r = np.sort(rng.uniform(0.1, 3, 2500))
        k = np.sort(rng.uniform(0.01, 0.95 * z / 3.0, ni))
    else:
        r = np.sort(rng.uniform(0.5, 50.0, 2500))
        k = np.sort(rng.uniform(0.01, 2.0, ni))
    m, n = len(r), len(k)
    c = np.asfortranarray(rng.standard_normal((m, B)))
    g0 = np.asfortranarray(rng.standard_normal((n, B)))
    g = g0.copy(order="F")
    lib.add_loc_batch(L.dptr(g), nu, L.dptr(r), L.dptr(c), L.dptr(k), m, n, K, B, m, n, None, None, None)
    gd = orc.direct_sum(abs(nu), r, k, c, np.arange(n))
    assert col_err(g - g0, gd, c).max() <= 1e-8, (nu, B, K)


def test_launch_counter_moves(cuda):
    from nufht_b200 import _lib as L
    from nufht_b200 import _pynufht as pn
    before = L.lib().nufht_b200_launch_count()
    r, k = grids("uniform", 3000, 3000, 40)
    pn.nufht_batch(0.0, r, np.ones((3000, 2)), k)
    assert L.lib().nufht_b200_launch_count() > before


def test_pynufht_plan_cache(cuda, orc):
    """Repeated nufht_batch calls on the same grids reuse one cached plan; other grids or
    tolerances get their own; results match the oracle every time."""
    from nufht_b200 import _pynufht as pn
    pn.clear_plan_cache()
    r, k = grids("uniform", 2500, 2000, 21)
    rng = np.random.default_rng(21)
    for q in range(3):
        c = rng.standard_normal((2500, 2))
        g = pn.nufht_batch(0.0, r, c, k, 1e-8)
        assert col_err(g, orc.nufht_batch(0.0, r, k, c, 1e-8), c).max() <= 1e-8
    assert len(pn._plans.entries) == 1
    pn.nufht_batch(0.0, r, c, k, 1e-6)
    pn.nufht_batch(1.0, r, c, k, 1e-8)
    assert len(pn._plans.entries) == 3
    pn.clear_plan_cache()
    assert not pn._plans.entries


def test_reference_c_program(cuda, orc, tmp_path):
    """The reference's own C test (src/test_nufht.c: nu = 1/2, f = (1 + r^2)^-n for n = 2, 3
    on 10000 Gauss-Legendre nodes in [0, 10], 100 k in (0, 10], tol 1e-8), compiled unchanged
    against the reference header and linked with libnufht_b200.so, runs on the GPU: its
    printed transform values agree with the oracle on the same inputs, and its errors against
    the analytic transforms are the oracle's (the truncation of the integral at r = 10)."""
    import subprocess
    from test_planner_abi import REF_OUT, write_gl_file
    exe = os.path.join(REF_OUT, "test_nufht_ref")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref was built without the reference tree")
    gl = str(tmp_path / "gl10000")
    write_gl_file(gl)
    out = subprocess.run([exe, gl], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    cols, cur = {}, None
    for ln in out.stdout.splitlines():
        if ln.startswith("# Batch column n="):
            cur = int(ln.split("=")[1])
            cols[cur] = []
        elif ln.strip() and not ln.startswith("#"):
            cols[cur].append([float(v) for v in ln.split()])
    assert sorted(cols) == [2, 3]
    # the same inputs as the program (src/test_nufht.c:47-88)
    x, w = np.loadtxt(gl, unpack=True)
    r, w = 5.0 * (x + 1.0), 5.0 * w
    c = np.stack([r ** 1.5 * (1 + r * r) ** -n * w for n in (2, 3)], axis=1)
    k = 10.0 * np.arange(1, 101) / 100
    g = orc.nufht_batch(0.5, r, k, c, 1e-8)
    for b, n in enumerate((2, 3)):
        a = np.array(cols[n])
        assert a.shape == (100, 4) and np.allclose(a[:, 0], k, rtol=1e-7)
        numeric_oracle = np.sqrt(np.pi / (2 * k)) * g[:, b]
        l1 = np.abs(c[:, b]).sum()
        # values are printed with 9 significant digits
        bound = 1e-8 * np.sqrt(np.pi / (2 * k)) * l1 + 1e-8 * np.abs(numeric_oracle)
        assert (np.abs(a[:, 2] - numeric_oracle) <= bound).all(), n
        err_oracle = np.abs(numeric_oracle - a[:, 1]).max()
        assert np.abs(a[:, 2] - a[:, 1]).max() <= err_oracle + 1e-7, (n, err_oracle)
