"""The C oracle against the golden fixtures of tests/golden (independent
NumPy/SciPy restatement).  CPU only."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "case_*.npz")))


def load(path):
    z = np.load(path, allow_pickle=False)
    g = O.Grid(z["xn"], z["yn"], z["zn"])
    return z, g


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(params=GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def case(request):
    return load(request.param)


def test_golden_present():
    assert len(GOLD) == 4


def test_sigma_hat(case):
    z, g = case
    s = O.sigma_hat(str(z["mode"]), float(z["omega"]), z["sig_re"], z["eps_rel"], z["eta"],
                    z["tau"], z["cee"])
    assert relerr(s, z["sig"]) < 1e-14


def test_k2(case):
    z, g = case
    k2 = O.gen_k2(g, z["sig"], float(z["omega"]))
    assert relerr(k2, z["k2"]) < 1e-14
    assert np.all(np.isfinite(k2))


def test_diag(case):
    z, g = case
    d = O.gen_diag(g, z["k2"])
    assert relerr(d, z["diag"]) < 1e-13


def test_inprod(case):
    z, g = case
    y = O.inprod(g, z["k2"], z["x"])
    assert relerr(y, z["y"]) < 1e-13


def test_rhs_mode5(case):
    z, g = case
    dips = [(str(d),) + tuple(int(v) for v in ijk) for d, ijk in zip(z["dip_dirs"], z["dip_ijk"])]
    b, nsk = O.gen_rhs(g, 5, dips)
    assert nsk == int(z["nskip"])
    assert relerr(b, z["rhs"]) < 1e-15


def test_qmr_history(case):
    z, g = case
    r = O.qmr(g, z["k2"], z["diag"], z["rhs"], 1e-10, 3000)
    hz = z["qmr_hist"]
    assert r["converged"] == bool(z["qmr_conv"])
    assert abs(r["iters"] - int(z["qmr_iters"])) <= 1
    m = min(len(hz), len(r["hist"]), 40)
    # relative agreement, with a floor at the recurrence's rounding level
    floor = 1e-12 * r["rhsnorm"]
    assert np.all(np.abs(r["hist"][:m] - hz[:m]) <= 1e-8 * hz[:m] + floor)
    # converged QMR against the sparse direct solve
    assert relerr(r["x"], z["sol_direct"]) < 1e-7


def test_fields(case):
    z, g = case
    B, E = O.gen_fields(g, float(z["omega"]), z["qmr_x"])
    assert relerr(B, z["fields_B"]) < 1e-13
    assert relerr(E, z["fields_E"]) < 1e-13


def test_qmr_threads_match(case):
    z, g = case
    r1 = O.qmr(g, z["k2"], z["diag"], z["rhs"], 1e-10, 3000, nthreads=1)
    r4 = O.qmr(g, z["k2"], z["diag"], z["rhs"], 1e-10, 3000, nthreads=4)
    assert r1["iters"] == r4["iters"]
    assert np.array_equal(r1["hist"], r4["hist"])
