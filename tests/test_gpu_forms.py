"""The alternative kernel forms the library keeps beside its default ones, run in fresh
processes (the switches are read once per process): the tensor-core direct kernel
(NUFHT_B200_DIR_MMA=1) and the SIMT local kernels (NUFHT_B200_LOC_SIMT=1) against the default
forms (SIMT direct, tensor-core local), the plain
per-plan term count (NUFHT_B200_TERM_SPLIT=0) against the per-box term split, and direct
Bessel evaluation (NUFHT_B200_DIR_NO_TABLE=1) against the J_nu table.  Every form is also
checked against the oracle."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, col_err, grids

pytestmark = pytest.mark.gpu

CASES = [(0.0, "loguniform", 20000, 15000, 1e-8), (3.0, "uniform", 12000, 9000, 1e-10),
         (10.0, "uniform", 3000, 4000, 1e-8)]

SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests/golden")
from make_golden import grids
from nufht_b200 import DevicePlan
import torch
out = {}
for q, (nu, kind, m, n, tol) in enumerate(%r):
    r, k = grids(kind, m, n, 40 + q)
    c = np.random.default_rng(q).standard_normal((m, 7))
    p = DevicePlan(nu, r, k, tol)
    out["g%%d" %% q] = p(torch.tensor(c, device="cuda")).cpu().numpy()
    p.close()
np.savez(sys.argv[2], **out)
""" % (CASES,)


def _run(tmp_path, name, env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    path = str(tmp_path / (name + ".npz"))
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT, path], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(path)


@pytest.fixture(scope="module")
def forms(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("forms")
    return {
        "default": _run(tmp, "default", {}),
        "alt": _run(tmp, "alt", {"NUFHT_B200_DIR_MMA": "1", "NUFHT_B200_LOC_SIMT": "1"}),
        "nosplit": _run(tmp, "nosplit", {"NUFHT_B200_TERM_SPLIT": "0"}),
        "notable": _run(tmp, "notable", {"NUFHT_B200_DIR_NO_TABLE": "1"}),
    }


@pytest.mark.parametrize("q", range(len(CASES)))
def test_kernel_forms_agree_and_match_the_oracle(cuda, orc, forms, q):
    nu, kind, m, n, tol = CASES[q]
    r, k = grids(kind, m, n, 40 + q)
    c = np.random.default_rng(q).standard_normal((m, 7))
    idx = np.random.default_rng(100 + q).choice(n, 300, replace=False)
    exact = orc.direct_sum(nu, r, k, c, idx)
    ref = forms["default"]["g%d" % q]
    for name, f in forms.items():
        g = f["g%d" % q]
        assert col_err(g[idx], exact, c).max() <= tol, (name, q)
        # the forms differ in summation order and tile shapes only (same expansions), except
        # the term split, whose dropped terms are below the tolerance by the switch table
        bar = tol if name == "nosplit" else 1e-13
        assert col_err(g, ref, c).max() <= bar, (name, q)
