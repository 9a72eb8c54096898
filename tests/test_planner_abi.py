"""Product library on the CPU side: exported C ABI, struct layouts, host planner and
parameter lookup against the reference's golden box lists and the oracle."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT, grids

HEADER = os.path.join(ROOT, "include", "nufht_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)
    skip = {"if", "while", "for", "return", "sizeof", "defined"}
    return sorted({n for n in names if n not in skip and not n.isupper()})


def test_library_exports_every_declared_symbol(plib):
    names = declared_functions()
    assert "nufht_batch" in names and "nufht_b200_execute" in names
    missing = [n for n in names if not hasattr(plib, n)]
    assert not missing, missing


def test_reference_globals_exported(plib):
    for g in ("ASY_COEF_TABLE", "ASY_Z_TABLE", "WIMP_K_TABLE"):
        assert ctypes.c_double.in_dll(plib, g) is not None


def test_struct_layouts_match_reference():
    """sizeof / offsetof of the reference structs on x86-64 (src/fast_hankel_nufht.h)."""
    from nufht_b200 import _lib as L
    assert ctypes.sizeof(L.NufhtOptions) == 32
    assert ctypes.sizeof(L.NufhtPlan) == 656
    assert ctypes.sizeof(L.NufhtScratch) == 72
    assert ctypes.sizeof(L.Box) == 16 and ctypes.sizeof(L.BoxVector) == 24 and ctypes.sizeof(L.Boxes) == 72
    assert L.NufhtPlan.m.offset == 544 and L.NufhtPlan.rs.offset == 552
    assert L.NufhtPlan.max_levels.offset == 568 and L.NufhtPlan.boxes.offset == 576
    assert L.NufhtPlan.tables_loaded.offset == 648


REF_OUT = os.path.join(ROOT, "oracle", "_ref")


def test_c_header_layouts_match_reference_header():
    """include/nufht_b200.h against the reference's own src/fast_hankel_nufht.h, in C: the
    build compiles oracle/abi_layout.c against each header, and the checking program only
    compiles when every struct size and field offset is equal (_Static_assert)."""
    import subprocess
    exe = os.path.join(REF_OUT, "abi_layout_check")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref was built without the reference tree")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=30)
    assert out.returncode == 0 and "matches the reference header: 47" in out.stdout, out.stdout


def write_gl_file(path, n=10000):
    """Gauss-Legendre nodes and weights on [-1, 1] in the reference's two-column data format
    (data/gl10000), computed with NumPy."""
    x, w = np.polynomial.legendre.leggauss(n)
    np.savetxt(path, np.c_[x, w], fmt="%.17e")


def test_reference_c_program_links_the_library(tmp_path):
    """The reference's src/test_nufht.c, compiled unchanged against its own header and linked
    with libnufht_b200.so, plans through the drop-in (nufht_plan_init, nufht_scratch_init) and
    reaches nufht_batch, which reports that there is no GPU here (the GPU test runs it)."""
    import subprocess
    from conftest import gpu_available
    exe = os.path.join(REF_OUT, "test_nufht_ref")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref was built without the reference tree")
    if gpu_available():
        pytest.skip("a GPU is present: covered by test_gpu_parity.py::test_reference_c_program")
    gl = str(tmp_path / "gl10000")
    write_gl_file(gl)
    out = subprocess.run([exe, gl], capture_output=True, text=True, timeout=120)
    assert "nufht_batch returned %d" % -422 in out.stderr, (out.stdout[-500:], out.stderr[-500:])


def test_default_options(plib):
    o = plib.nufht_default_options()
    assert o.tol == 1e-8 and o.max_levels == 0 and o.min_dim_prod == 10000
    assert math.isnan(o.z_split) and o.K_asy == 0 and o.K_loc == 0


@pytest.mark.parametrize("q", range(7))
def test_generate_boxes_matches_reference(plib, golden, q):
    from nufht_b200 import _lib as L
    b = golden("boxes_golden.npz")
    m, n, seed, nu, tol, z, ka, kl = b["case%d_meta" % q]
    r, k = grids(str(b["case%d_kind" % q]), int(m), int(n), int(seed))
    bx = plib.generate_boxes(r.ctypes.data_as(L.c_double_p), int(m), k.ctypes.data_as(L.c_double_p), int(n),
                             float(z), 0, 10000, int(kl))
    loc, asy, dr = L.boxes_to_array(bx)
    plib.boxes_free(ctypes.byref(bx))
    np.testing.assert_array_equal(loc, b["case%d_loc" % q])
    np.testing.assert_array_equal(asy, b["case%d_asy" % q])
    np.testing.assert_array_equal(dr, b["case%d_dir" % q])


@pytest.mark.parametrize("seed", range(12))
def test_plan_init_matches_oracle_random(plib, orc, seed):
    """Random sizes, orders, tolerances and grids with ties: the plan's parameters and boxes
    equal the restated reference planner's."""
    from nufht_b200 import _lib as L
    rng = np.random.default_rng(1000 + seed)
    m, n = int(rng.integers(1, 4000)), int(rng.integers(1, 4000))
    nu = float(rng.choice([0, 1, 2, 3, 7, 10, 34, 35, 100, -1, -4, 0.5, 2.5, -1.5]))
    tol = float(10.0 ** -rng.integers(4, 16))
    r = np.sort(np.round(rng.uniform(0, 1, m) * 300, 1)) + 0.05
    k = np.sort(10 ** rng.uniform(-2, 2.5, n))
    opt = L.options(tol=tol)
    plan = L.NufhtPlan()
    rc = plib.nufht_plan_init(ctypes.byref(plan), nu, L.dptr(r), m, L.dptr(k), n, ctypes.byref(opt))
    orc_rc, z, ka, kl, coef = orc.plan_params(nu, tol)
    assert rc == orc_rc == 0
    assert plan.K_asy == ka and plan.K_loc == kl
    assert (math.isnan(plan.z_split) and math.isnan(z)) or plan.z_split == z
    np.testing.assert_array_equal(np.array(plan.asy_coef[:]), coef)
    got = L.boxes_to_array(plan.boxes)
    if not math.isnan(z):
        want = orc.boxes(r, k, z, 0, 10000, max(kl, 0))
        for a, w in zip(got, want):
            np.testing.assert_array_equal(a, w)
    plib.nufht_plan_free(ctypes.byref(plan))


def test_plan_init_error_codes(plib):
    from nufht_b200 import _lib as L
    r = np.linspace(0.1, 10, 50)
    k = np.linspace(0.1, 5, 40)
    plan = L.NufhtPlan()

    def init(nu, rr=r, kk=k, tol=1e-8, m=None, n=None):
        opt = L.options(tol=tol)
        rc = plib.nufht_plan_init(ctypes.byref(plan), nu, L.dptr(rr), len(rr) if m is None else m, L.dptr(kk),
                                  len(kk) if n is None else n, ctypes.byref(opt))
        plib.nufht_plan_free(ctypes.byref(plan))
        return rc

    assert init(0.0) == 0
    assert init(0.0, tol=1e-16) == -1
    assert init(0.25) == -2
    assert init(200.5) == -2
    assert init(10.5) == -2
    assert init(-201.0) == -2
    assert init(0.0, m=0) == -200
    assert init(0.0, n=-1) == -200
    assert plib.nufht_plan_init(None, 0.0, L.dptr(r), 50, L.dptr(k), 40, None) == -200
    assert init(0.0, rr=r[::-1].copy()) == L.NUFHT_E_UNSORTED_RS
    assert init(0.0, kk=np.r_[k[:-1], np.nan]) == L.NUFHT_E_UNSORTED_WS
    assert init(0.0, rr=np.r_[-1.0, r[1:]]) == L.NUFHT_E_UNSORTED_RS


def test_batch_argument_errors_without_gpu(plib):
    from nufht_b200 import _lib as L
    r = np.linspace(0.1, 10, 50)
    k = np.linspace(0.1, 5, 40)
    plan = L.NufhtPlan()
    assert plib.nufht_plan_init(ctypes.byref(plan), 0.0, L.dptr(r), 50, L.dptr(k), 40, None) == 0
    c = np.zeros((50, 2), order="F")
    g = np.zeros((40, 2), order="F")
    assert plib.nufht_batch(ctypes.byref(plan), None, 50, L.dptr(g), 40, 2, None) == -400
    assert plib.nufht_batch(ctypes.byref(plan), L.dptr(c), 50, L.dptr(g), 40, 0, None) == -400
    assert plib.nufht_batch(ctypes.byref(plan), L.dptr(c), 49, L.dptr(g), 40, 2, None) == -401
    assert plib.nufht_batch(ctypes.byref(plan), L.dptr(c), 50, L.dptr(g), 39, 2, None) == -401
    plib.nufht_plan_free(ctypes.byref(plan))


def test_scratch_sizes_follow_reference(plib):
    from nufht_b200 import _lib as L
    r = np.linspace(0.1, 10, 500)
    k = np.linspace(0.1, 50, 400)
    plan = L.NufhtPlan()
    assert plib.nufht_plan_init(ctypes.byref(plan), 7.0, L.dptr(r), 500, L.dptr(k), 400, None) == 0
    s = L.NufhtScratch()
    assert plib.nufht_scratch_init(ctypes.byref(s), ctypes.byref(plan)) == 0
    assert s.m_alloc == 500 and s.n_alloc == 400 and s.Kloc_alloc == plan.K_loc and s.extra_alloc == 4
    plib.nufht_scratch_free(ctypes.byref(s))
    assert plib.nufht_scratch_init(None, ctypes.byref(plan)) == -300
    plib.nufht_plan_free(ctypes.byref(plan))


def test_split_box_matches_oracle(plib, orc):
    from nufht_b200 import _lib as L
    r, k = grids("uniform", 5000, 4000, 9)
    rc, z, ka, kl, _ = orc.plan_params(0.0, 1e-8)
    box = L.Box(100, 3500, 200, 4800)
    i = ctypes.c_int()
    j = ctypes.c_int()
    plib.split_box(r.ctypes.data_as(L.c_double_p), 5000, k.ctypes.data_as(L.c_double_p), 4000,
                   ctypes.byref(box), z, ctypes.byref(i), ctypes.byref(j))
    # the split row maximises the loc+asy area over 10 candidates (src/fast_hankel_nufht.c:498-574)
    cand = sorted(set(int(round(100 + t / 9 * 3400)) for t in range(10)))
    def obj(ii):
        jj = int(np.searchsorted(r, z / k[ii], side="right"))
        return (ii - 100 + 1) * (jj - 200 + 1) + (3500 - ii + 1) * (4800 - jj + 1)
    best = max(cand, key=lambda c: (obj(c), -c))
    assert i.value == best and j.value == int(np.searchsorted(r, z / k[best], side="right"))


def test_pynufht_shape_errors():
    from nufht_b200 import _pynufht as pn
    r = np.linspace(0.1, 1, 10)
    k = np.linspace(0.1, 1, 5)
    with pytest.raises(ValueError, match="2-D"):
        pn.nufht_batch(0.0, r, np.zeros(10), k)
    with pytest.raises(ValueError, match="first dimension"):
        pn.nufht_batch(0.0, r, np.zeros((9, 2)), k)
    with pytest.raises(ValueError, match="2-D"):
        pn.nufht_batch_loop(0.0, r, np.zeros(10), k)


def test_table_generator_matches_reference_generator():
    """generate_tables() of the library fills the exported globals with the values of the
    reference's own generator (oracle/_ref, when built here) or the golden rows."""
    import oracle
    from nufht_b200 import _lib as L
    lib = L.lib()
    lib.generate_tables()
    z = np.ctypeslib.as_array((ctypes.c_double * (401 * 32 * 16)).in_dll(lib, "ASY_Z_TABLE")).reshape(401, 32, 16)
    kw = np.ctypeslib.as_array((ctypes.c_int * (401 * 32 * 16)).in_dll(lib, "WIMP_K_TABLE")).reshape(401, 32, 16)
    f = open(oracle.TABLES, "rb").read()
    z2 = np.frombuffer(f, np.float64, 401 * 32 * 16, 24 + 401 * 64 * 8).reshape(401, 32, 16)
    np.testing.assert_array_equal(z, z2)
    assert kw[0, 4, 3] == 14 and abs(z[0, 4, 3] - 10.9099) < 1e-3
