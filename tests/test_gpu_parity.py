"""GPU parity of the complex128 path against the CPU oracle, through the C ABI.

Tolerances: FP64 arithmetic with different summation order and FMA
contraction, so operator outputs agree to 1e-13 relative (norm-wise per
vector); QMR residual histories agree to 1e-9 relative over the first 40
iterations; iteration counts agree exactly or within one iteration where the
stop test sits on a rounding boundary.
"""
import glob
import os

import numpy as np
import pytest

from aphid_git_b200 import Solver, model
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "case_*.npz")))


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def solver():
    s = Solver(graph_iters=8)
    yield s
    s.close()


def random_grid(rng, dims):
    return [np.cumsum(np.concatenate([[0.0], rng.uniform(50.0, 400.0, n - 1)])) for n in dims]


def mesh_case(solver, rng, dims, freq=3.0, mode="R"):
    xn, yn, zn = random_grid(rng, dims)
    g = O.Grid(xn, yn, zn)
    solver.set_nodes(xn, yn, zn)
    cs = tuple(d - 1 for d in dims)
    sig_re = (10.0 ** rng.uniform(-4, 1, cs)).astype(np.float32)
    sig_re[:, :, :2] = 1e-8
    w = 2 * np.pi * freq
    sig = O.sigma_hat(mode, w, sig_re, eps_rel=rng.uniform(1, 20, cs))
    k2 = O.gen_k2(g, sig, w)
    return g, sig, w, k2


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_golden_operator_chain(solver, path):
    z = np.load(path)
    g = O.Grid(z["xn"], z["yn"], z["zn"])
    solver.set_nodes(z["xn"], z["yn"], z["zn"])
    w = float(z["omega"])
    k2 = solver.gen_k2(z["sig"], w)
    assert relerr(k2, z["k2"]) < 1e-14
    assert relerr(solver.gen_diag(z["k2"]), z["diag"]) < 1e-13
    assert relerr(solver.inprod(z["k2"], z["x"]), z["y"]) < 1e-13
    B, E = solver.gen_fields(w, z["qmr_x"])
    assert relerr(B, z["fields_B"]) < 1e-13 and relerr(E, z["fields_E"]) < 1e-13


@pytest.mark.parametrize("dims", [(5, 4, 3), (33, 17, 9), (40, 37, 29)])
def test_inprod_random(solver, dims):
    rng = np.random.default_rng(sum(dims))
    g, sig, w, k2 = mesh_case(solver, rng, dims)
    x = rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n)
    y0 = O.inprod(g, k2, x)
    y1 = solver.inprod(k2, x)
    off = model.block_offsets(*g.dims)
    for b in range(4):
        sl = slice(off[b], off[b + 1])
        assert relerr(y1[sl], y0[sl]) < 1e-13, b
    assert relerr(solver.gen_k2(sig, w), k2) < 1e-14
    assert relerr(solver.gen_diag(k2), O.gen_diag(g, k2)) < 1e-13


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_qmr_golden(solver, path):
    z = np.load(path)
    g = O.Grid(z["xn"], z["yn"], z["zn"])
    solver.set_nodes(z["xn"], z["yn"], z["zn"])
    ref = O.qmr(g, z["k2"], z["diag"], z["rhs"], 1e-10, 3000)
    x, info, hist = solver.qmr(z["k2"], z["diag"], z["rhs"], 1e-10, 3000)
    assert info["status_name"] == "converged"
    assert abs(info["iters"] - ref["iters"]) <= 1
    m = min(40, len(hist), len(ref["hist"]))
    floor = 1e-12 * ref["rhsnorm"]
    assert np.all(np.abs(hist[:m] - ref["hist"][:m]) <= 1e-9 * ref["hist"][:m] + floor)
    assert relerr(x, ref["x"]) < 1e-8
    assert relerr(x, z["sol_direct"]) < 1e-7
    assert info["true_rel_resid"] < 1e-9


def test_qmr_halfspace32_matches_oracle(solver):
    m = model.make_model("halfspace32")
    g = O.Grid(m.xn, m.yn, m.zn)
    solver.set_nodes(m.xn, m.yn, m.zn)
    w = 2 * np.pi * m.freqs[0]
    sig = model.sigma_hat("R", w, m.sig_re.ravel(order="F"))
    k2 = solver.gen_k2(sig, w)
    diag = solver.gen_diag(k2)
    b, _ = model.gen_rhs(m.xn, m.yn, m.zn, 5, m.sources[0])
    ref = O.qmr(g, k2, diag, b, 1e-8, 5000)
    x, info, hist = solver.qmr(k2, diag, b, 1e-8, 5000)
    assert ref["converged"] and info["status_name"] == "converged"
    assert abs(info["iters"] - ref["iters"]) <= max(1, ref["iters"] // 50)
    assert relerr(x, ref["x"]) < 1e-6
    # fields of the two solutions
    B0, E0 = O.gen_fields(g, w, ref["x"])
    B1, E1 = solver.gen_fields(w, x)
    assert relerr(E1, E0) < 1e-6 and relerr(B1, B0) < 1e-6


def test_qmr_iteration_cap_semantics(solver):
    z = np.load(GOLD[0])
    g = O.Grid(z["xn"], z["yn"], z["zn"])
    solver.set_nodes(z["xn"], z["yn"], z["zn"])
    for max_it in (0, 1, 2, 7):
        ref = O.qmr(g, z["k2"], z["diag"], z["rhs"], 1e-30, max_it)
        x, info, hist = solver.qmr(z["k2"], z["diag"], z["rhs"], 1e-30, max_it)
        assert info["iters"] == ref["iters"], max_it
        assert info["status_name"] == "maxit"
        assert len(hist) == len(ref["hist"]) == max(1, max_it)
        assert relerr(x, ref["x"]) < 1e-10


def test_qmr_initial_guess(solver):
    z = np.load(GOLD[1])
    g = O.Grid(z["xn"], z["yn"], z["zn"])
    solver.set_nodes(z["xn"], z["yn"], z["zn"])
    x0 = z["sol_direct"] * (1 + 1e-3)
    ref = O.qmr(g, z["k2"], z["diag"], z["rhs"], 1e-10, 3000, x0=x0)
    x, info, _ = solver.qmr(z["k2"], z["diag"], z["rhs"], 1e-10, 3000, x0=x0)
    assert abs(info["iters"] - ref["iters"]) <= 1
    assert info["iters"] < int(z["qmr_iters"])
    assert relerr(x, z["sol_direct"]) < 1e-7


def test_qmr_zero_rhs_reports_breakdown(solver):
    z = np.load(GOLD[0])
    solver.set_nodes(z["xn"], z["yn"], z["zn"])
    x, info, _ = solver.qmr(z["k2"], z["diag"], np.zeros_like(z["rhs"]), 1e-10, 100)
    assert info["status_name"] == "breakdown"
    assert np.all(x == 0)


def test_qmr_boundary_source_never_converges(solver):
    # a source on a boundary node meets a zero row of K: the reference
    # iterates to qmr_max_it; the GPU path stops with the same count or
    # reports the breakdown the recurrence runs into.
    z = np.load(GOLD[0])
    g = O.Grid(z["xn"], z["yn"], z["zn"])
    solver.set_nodes(z["xn"], z["yn"], z["zn"])
    nx, ny, nz = g.dims
    b, _ = model.gen_rhs(z["xn"], z["yn"], z["zn"], 5, [("+Z", 2, 2, 1)])
    x, info, hist = solver.qmr(z["k2"], z["diag"], b, 1e-10, 60)
    assert info["status_name"] in ("maxit", "breakdown", "nonfinite")
    assert info["true_rel_resid"] > 1e-3 or not np.isfinite(info["true_rel_resid"])


def test_qmr_deterministic(solver):
    z = np.load(GOLD[2])
    solver.set_nodes(z["xn"], z["yn"], z["zn"])
    a = solver.qmr(z["k2"], z["diag"], z["rhs"], 1e-10, 3000)
    b = solver.qmr(z["k2"], z["diag"], z["rhs"], 1e-10, 3000)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])


def test_bad_arguments_raise(solver):
    from aphid_git_b200 import AphidError
    z = np.load(GOLD[0])
    solver.set_nodes(z["xn"], z["yn"], z["zn"])
    with pytest.raises(AphidError):
        solver.qmr(z["k2"], z["diag"], z["rhs"], -1.0, 10)
    with pytest.raises(AphidError):
        solver.set_mesh(np.zeros(4), np.ones(4), np.ones(4), np.ones(3), np.ones(3), np.ones(3))
