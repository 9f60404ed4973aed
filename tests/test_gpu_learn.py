"""What the learned initial guess gains over the zero start, on an unseen
model of the training generator, through the same complex128 QMR (the
reference's recurrence) from both starts.  The shipped network's guesses do
not pay on these problems (their fitted residual stays near ||b||), so the
guard drops them and the count is the zero-start count: the test pins that
the learned path never costs iterations and never changes the answer, and
that an accepted guess is used (a near-exact guess saves most of the
iterations)."""
import numpy as np
import pytest

from aphid_git_b200 import Solver, learn, model

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    m = model.make_model("train64", seed=77)
    s = Solver()
    s.set_nodes(m.xn, m.yn, m.zn)
    yield m, s
    s.close()


def _system(s, m, f):
    w = 2 * np.pi * f
    k2 = s.gen_k2(model.sigma_hat("R", w, m.sig_re.ravel(order="F")), w)
    b, _ = model.gen_rhs(m.xn, m.yn, m.zn, 5, m.sources[0])
    return k2, s.gen_diag(k2), b


@pytest.mark.parametrize("f", [0.1, 30.0])
def test_learned_guess_never_costs_iterations(case, f):
    m, s = case
    p = learn.load_params()
    assert p is not None and p.size == 1463896
    g = learn.Guess(p, m.dims)
    try:
        x0, r0 = g.x0(s, m.sig_re, f, m.sources[0])
    finally:
        g.close()
    k2, dg, b = _system(s, m, f)
    x_zero, i_zero, _ = s.qmr(k2, dg, b, 1e-8, 20000)
    x_nn, i_nn, _ = s.qmr(k2, dg, b, 1e-8, 20000, x0=x0)
    gain = i_zero["iters"] - i_nn["iters"]
    print("f=%g: zero start %d iterations, learned %d (gain %d), guess residual %.3f, used %s"
          % (f, i_zero["iters"], i_nn["iters"], gain, r0, x0 is not None))
    assert i_nn["status_name"] == "converged"
    assert gain >= 0
    assert np.linalg.norm(x_nn - x_zero) <= 1e-6 * np.linalg.norm(x_zero)


def test_an_accepted_guess_is_used(case):
    m, s = case
    f = 1.0
    k2, dg, b = _system(s, m, f)
    x, i_zero, _ = s.qmr(k2, dg, b, 1e-10, 20000)
    # a near-exact guess in the network's output form, through the same fit
    y = learn.compress(learn.pack_solution(x, m.dims))
    groups = learn.unpack_groups(learn.expand(y), m.dims)
    x0, alpha = learn.fit_amplitudes(s, k2, b, groups)
    r0 = np.linalg.norm(b - s.inprod(k2, x0)) / np.linalg.norm(b)
    assert r0 < learn.ACCEPT
    _, i_nn, _ = s.qmr(k2, dg, b, 1e-8, 20000, x0=x0)
    _, i_z8, _ = s.qmr(k2, dg, b, 1e-8, 20000)
    assert i_nn["iters"] < i_z8["iters"] / 2
