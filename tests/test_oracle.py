"""The CPU oracle (test infrastructure) pinned against the golden fixtures and the
reference's own known-answer tests."""
import math

import numpy as np
import pytest

from conftest import col_err, grids


def test_oracle_bessel_vs_mpmath(orc, golden):
    g = golden("bessel_golden.npz")
    got = np.array([orc.besselj(nu, x)[0] for nu, x in zip(g["nu"], g["x"])])
    err = np.abs(got - g["j"])
    assert err.max() < 2e-15, (err.max(), g["nu"][err.argmax()], g["x"][err.argmax()])


def test_oracle_tables_match_reference_cache(orc, golden):
    """The oracle reads the library-generated cache; its rows agree with the reference's
    shipped cache (coefficients and Wimp degrees exactly, switch points to Newton noise)."""
    t = golden("tables_golden.npz")
    from nufht_b200 import _lib  # noqa: F401  (table cache is produced by the library build)
    import oracle
    f = open(oracle.TABLES, "rb").read()
    coef = np.frombuffer(f, np.float64, 401 * 64, 24).reshape(401, 64)
    z = np.frombuffer(f, np.float64, 401 * 32 * 16, 24 + 401 * 64 * 8).reshape(401, 32, 16)
    kw = np.frombuffer(f, np.int32, 401 * 32 * 16, 24 + 401 * 64 * 8 + 401 * 32 * 16 * 8).reshape(401, 32, 16)
    for row, ref in zip(t["coef_rows"], t["coef"]):
        np.testing.assert_array_equal(coef[row], ref)
    for q, nu in enumerate(t["nus"]):
        np.testing.assert_array_equal(kw[nu, :12, :11], t["kw"][q])
        np.testing.assert_allclose(z[nu, :12, :11], t["z"][q], atol=3e-4, rtol=0)


@pytest.mark.parametrize("q", range(7))
def test_oracle_boxes_match_reference(orc, golden, q):
    b = golden("boxes_golden.npz")
    meta = b["case%d_meta" % q]
    m, n, seed, nu, tol, z, ka, kl = meta
    r, k = grids(str(b["case%d_kind" % q]), int(m), int(n), int(seed))
    loc, asy, dr = orc.boxes(r, k, z, 0, 10000, int(kl))
    np.testing.assert_array_equal(loc, b["case%d_loc" % q])
    np.testing.assert_array_equal(asy, b["case%d_asy" % q])
    np.testing.assert_array_equal(dr, b["case%d_dir" % q])


@pytest.mark.parametrize("nu,tol", [(0.0, 1e-8), (1.0, 1e-6), (10.0, 1e-12), (35.0, 1e-8), (0.5, 1e-8),
                                    (9.5, 1e-4), (-3.0, 1e-10)])
def test_oracle_plan_params(orc, golden, nu, tol):
    rc, z, ka, kl, coef = orc.plan_params(nu, tol)
    assert rc == 0
    if float(nu).is_integer():
        assert ka == min(int(math.floor(abs(nu) / 5 + math.log10(1 / tol) / 4 + 1)), 10)
    else:
        assert ka == int(round(abs(nu) - 0.5)) and kl == -1 and math.isnan(z)


def test_oracle_param_errors(orc):
    assert orc.plan_params(0.0, 1e-16)[0] == -1
    assert orc.plan_params(0.3, 1e-8)[0] == -2
    assert orc.plan_params(201.0, 1e-8)[0] == -2
    assert orc.plan_params(10.5, 1e-8)[0] == -2


def test_oracle_e2e_reproduces_reference_driver(orc, golden):
    """oracle_nufht_batch (restated driver + planner) equals the reference's own driver and
    planner over the same evaluators, bit for bit."""
    e = golden("e2e_golden.npz")
    for name in e["names"]:
        nu, tol, B = e[name + "_meta"]
        g = orc.nufht_batch(nu, e[name + "_r"], e[name + "_k"], e[name + "_c"], tol)
        np.testing.assert_array_equal(g, e[name + "_g"], err_msg=str(name))


def test_oracle_vs_direct_sum(orc, golden):
    e = golden("e2e_golden.npz")
    for name in e["names"]:
        nu, tol, B = e[name + "_meta"]
        if float(nu) == 0.5:
            continue  # half-integer path is checked in its own test
        r, k, c = e[name + "_r"], e[name + "_k"], e[name + "_c"]
        idx = np.arange(0, len(k), 37)
        d = orc.direct_sum(nu, r, k, c, idx)
        assert col_err(e[name + "_g"][idx], d, c).max() < tol, name


def test_oracle_type3_nufft_accuracy(orc):
    rng = np.random.default_rng(0)
    x = np.sort(rng.uniform(3, 50, 400))
    s = np.sort(rng.uniform(2, 40, 300))
    c = rng.standard_normal((3, 400)) + 1j * rng.standard_normal((3, 400))
    fe = orc.type3(x, c, s, mode=orc.T3_EXACT)
    for eps in (1e-6, 1e-8, 1e-10, 1e-12):
        fn = orc.type3(x, c, s, eps=eps, mode=orc.T3_NUFFT)
        assert (np.abs(fn - fe).max(axis=1) / np.abs(c).sum(axis=1)).max() < eps


def test_known_answer_gaussian_nu0(orc):
    """python/run_pynufht_test.py: nu = 0, c = r exp(-r^2/2) w on 1000 GL nodes on [0,10];
    the transform is exp(-k^2/2).  The reference's notebook records max abs errors ~1e-13
    (notebooks/nufht_batch_example.ipynb:190)."""
    x, w = np.polynomial.legendre.leggauss(1000)
    r, w = 5 * (x + 1), 5 * w
    cs = r * np.exp(-0.5 * r * r) * w
    k = 10 * np.arange(1, 101) / 100
    for mode in (orc.T3_EXACT, orc.T3_NUFFT):
        g = orc.nufht_batch(0.0, r, k, cs[:, None], 1e-8, mode=mode)[:, 0]
        assert np.abs(g - np.exp(-0.5 * k * k)).max() < 2e-13


def test_known_answer_half_integer(orc):
    """src/test_nufht.c: nu = 1/2, c = r^{3/2} (1+r^2)^{-n} w on 10000 GL nodes on [0,10];
    sqrt(pi/2k) G = (pi/4) e^{-k} (n=2), (pi/16)(1+k) e^{-k} (n=3) up to the truncation of
    the integral at r = 10, which dominates for small k."""
    x, w = np.polynomial.legendre.leggauss(10000)
    r, w = 5 * (x + 1), 5 * w
    cs = np.stack([r ** 1.5 * (1 + r * r) ** -n * w for n in (2, 3)], 1)
    k = 10 * np.arange(1, 101) / 100
    g = orc.nufht_batch(0.5, r, k, cs, 1e-8, mode=orc.T3_NUFFT)
    num = np.sqrt(np.pi / (2 * k))[:, None] * g
    an = np.stack([np.pi / 4 * np.exp(-k), np.pi / 16 * (1 + k) * np.exp(-k)], 1)
    # the tail of the integral beyond r = 10, bounded by int_10^inf r^{3/2-2n} sqrt(2/(pi k r))... * sqrt(pi/2k)
    tail = np.stack([10.0 ** (2 - 2 * n) / (2 * n - 2) / k for n in (2, 3)], 1)
    assert np.all(np.abs(num - an) <= tail + 1e-9)
    g_exact = orc.nufht_batch(0.5, r, k, cs, 1e-8, mode=orc.T3_EXACT)
    assert np.abs(g - g_exact).max() < 1e-8 * np.abs(cs).sum(axis=0).max()


def test_faithful_mode_keeps_reference_double_negation(orc):
    r, k = grids("uniform", 300, 200, 7)
    c = np.random.default_rng(1).standard_normal((300, 1))
    g1 = orc.nufht_batch(-1.0, r, k, c, 1e-8, faithful=True)
    g2 = orc.nufht_batch(-1.0, r, k, c, 1e-8, faithful=False)
    gp = orc.nufht_batch(1.0, r, k, c, 1e-8)
    np.testing.assert_array_equal(g1, gp)      # reference: batch==1 negated twice
    np.testing.assert_array_equal(g2, -gp)     # J_{-1} = -J_1
