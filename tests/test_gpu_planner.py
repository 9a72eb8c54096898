"""The device planner (box partition of the (k, r) rectangle on the GPU) against the golden box
lists of the reference's own generate_boxes, against the host planner at the full sizes of
the 1e6-point and 4e6-point workloads, on random grids with ties, and its input validation.
The lists must be identical, box for box and in order."""
import ctypes

import numpy as np
import pytest

from conftest import grids

pytestmark = pytest.mark.gpu


def _device_boxes(r, k, z, kl, max_levels=0, mdp=10000):
    from nufht_b200 import _lib as L
    lib = L.lib()
    out = L.Boxes()
    rc = lib.nufht_b200_generate_boxes_device(L.dptr(r), len(r), L.dptr(k), len(k), float(z), max_levels, mdp,
                                              int(kl), ctypes.byref(out))
    assert rc == 0, L.strerror(rc)
    arr = L.boxes_to_array(out)
    lib.boxes_free(ctypes.byref(out))
    return arr


def _host_boxes(r, k, z, kl, max_levels=0, mdp=10000):
    from nufht_b200 import _lib as L
    lib = L.lib()
    bx = lib.generate_boxes(r.ctypes.data_as(L.c_double_p), len(r), k.ctypes.data_as(L.c_double_p), len(k), float(z),
                            max_levels, mdp, int(kl))
    arr = L.boxes_to_array(bx)
    lib.boxes_free(ctypes.byref(bx))
    return arr


@pytest.mark.parametrize("q", range(7))
def test_device_partition_matches_reference_golden(cuda, golden, q):
    b = golden("boxes_golden.npz")
    m, n, seed, nu, tol, z, ka, kl = b["case%d_meta" % q]
    r, k = grids(str(b["case%d_kind" % q]), int(m), int(n), int(seed))
    loc, asy, dr = _device_boxes(r, k, z, kl)
    np.testing.assert_array_equal(loc, b["case%d_loc" % q])
    np.testing.assert_array_equal(asy, b["case%d_asy" % q])
    np.testing.assert_array_equal(dr, b["case%d_dir" % q])


def test_device_partition_full_size_workloads(cuda, orc):
    """N = M = 1e6 uniform on (0, 1000] at tol 1e-6 / 1e-8 / 1e-10 (both directions) and the
    4e6-point stress grids at order 100 (extended tables' split): device == host."""
    rng = np.random.default_rng(1)
    r = np.sort(1000.0 * (1.0 - rng.random(1_000_000)))
    k = np.sort(1000.0 * (1.0 - rng.random(1_000_000)))
    for tol in (1e-6, 1e-8, 1e-10):
        rc, z, ka, kl, coef = orc.plan_params(0.0, tol)
        for a, b in ((r, k), (k, r)):
            dev = _device_boxes(a, b, z, kl)
            host = _host_boxes(a, b, z, kl)
            for d, h in zip(dev, host):
                np.testing.assert_array_equal(d, h)
    rng = np.random.default_rng(100)
    n = 4_000_000
    means = np.array([200.0, 800.0, 1500.0])
    rr = np.sort(np.clip(np.abs(rng.normal(means[rng.integers(0, 3, n)], 50.0)), 1e-9, 2000.0))
    kk = np.sort(2000.0 * (1.0 - rng.random(n)))
    for z in (35.0, 152.7):
        for a, b in ((rr, kk), (kk, rr)):
            dev = _device_boxes(a, b, z, 120)
            host = _host_boxes(a, b, z, 120)
            for d, h in zip(dev, host):
                np.testing.assert_array_equal(d, h)


@pytest.mark.parametrize("seed", range(10))
def test_device_partition_random_grids_with_ties(cuda, seed):
    rng = np.random.default_rng(500 + seed)
    m, n = int(rng.integers(1, 30000)), int(rng.integers(1, 30000))
    r = np.sort(np.round(rng.uniform(0, 1, m) * 300, 1)) + 0.05 * (seed % 2)
    k = np.sort(10 ** rng.uniform(-2, 2.5, n))
    z = float(rng.uniform(2.0, 40.0))
    kl = int(rng.integers(0, 30))
    mdp = int(rng.choice([100, 1000, 10000]))
    lev = int(rng.choice([0, 3]))
    dev = _device_boxes(r, k, z, kl, lev, mdp)
    host = _host_boxes(r, k, z, kl, lev, mdp)
    for d, h in zip(dev, host):
        np.testing.assert_array_equal(d, h)


def test_device_planner_validates_grids_and_plans_record_it(cuda):
    from nufht_b200 import DevicePlan
    from nufht_b200 import _lib as L
    lib = L.lib()
    r = np.array([1.0, 2.0, 1.5, 3.0])
    k = np.linspace(0.1, 2.0, 5)
    out = L.Boxes()
    assert lib.nufht_b200_generate_boxes_device(L.dptr(r), 4, L.dptr(k), 5, 5.0, 0, 10, 0,
                                                ctypes.byref(out)) == L.NUFHT_E_UNSORTED_RS
    assert lib.nufht_b200_generate_boxes_device(L.dptr(k), 5, L.dptr(np.array([0.0, np.nan])), 2, 5.0, 0, 10, 0,
                                                ctypes.byref(out)) == L.NUFHT_E_UNSORTED_WS
    rng = np.random.default_rng(2)
    rr = np.sort(300.0 * rng.random(50000))
    kk = np.sort(100.0 * rng.random(40000))
    p = DevicePlan(0.0, rr, kk, 1e-8)
    st = p.stats()
    assert st[18] == 1.0 and st[15] > 0.0 and st[16] >= 0.0 and st[17] > 0.0
    host = _host_boxes(rr, kk, p.info()["z_split"], p.info()["K_loc"])
    b = p.boxes()
    nl, na = len(host[0]), len(host[1])
    np.testing.assert_array_equal(b[:nl], host[0])
    np.testing.assert_array_equal(b[nl:nl + na], host[1])
    np.testing.assert_array_equal(b[nl + na:], host[2])
    p.close()
