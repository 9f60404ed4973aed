"""Why AUTO escalates: the bilinear form of complex-symmetric Lanczos on the
reference's own operator (oracle, complex128), CPU only.

The complex-symmetric QMR of src/aphid_qmr.f90:297-372 normalises v~ in the
Hermitian norm and divides by delta = v~^T v~.  On a 96^3 mesh with 15 layers
of 3.3 S/m seawater under air, |delta| / ||v~||^2 falls below 1e-6 (the
escalation threshold of the sweep, kDeltaFloor) within a few dozen
iterations, at 0.27 Hz; complex64 storage perturbs v~^T v~ by about 6e-8
||v~||^2 and cannot carry the process past that point.  On the heterogeneous
land model of the same size (hetero96, 1 Hz), where the mixed-precision sweep
converges, it stays above 1e-5.
"""
import numpy as np

from aphid_git_b200 import model
from oracle import oracle as O

DELTA_FLOOR = 1e-6  # kDeltaFloor in aphid_git_b200/csrc/aphid_sweep.cuh


def min_bilinear_form(xn, yn, zn, sig, dipole, f, iters):
    """smallest |v~_n^T v~_n| (||v~_n|| = 1) over `iters` Lanczos steps of the
    Jacobi-scaled operator D^-1/2 K D^-1/2 from b"""
    g = O.Grid(xn, yn, zn)
    b, _ = O.gen_rhs(g, 5, [dipole])
    w = 2 * np.pi * f
    k2 = O.gen_k2(g, O.sigma_hat("R", w, sig_re=np.asarray(sig, np.float32).ravel(order="F")), w)
    s = 1.0 / np.sqrt(O.gen_diag(g, k2))
    v = s * b
    rho = np.linalg.norm(v)
    v = v / rho
    p = np.zeros_like(v)
    eps, delta = 1.0, v @ v
    dmin = abs(delta)
    for _ in range(iters):
        p = v - (rho * delta / eps) * p
        q = s * O.inprod(g, k2, s * p)
        eps = p @ q
        vt = q - (eps / delta) * v
        rho = np.linalg.norm(vt)
        v = vt / rho
        delta = v @ v
        dmin = min(dmin, abs(delta))
    return dmin


def test_seafloor_collapses_the_form_and_land_does_not():
    m = model.make_model("seafloor96")
    sea = min_bilinear_form(m.xn, m.yn, m.zn, m.sig_re, m.sources[0][0], 0.272, 80)
    h = model.make_model("hetero96")
    land = min_bilinear_form(h.xn, h.yn, h.zn, h.sig_re, h.sources[0][0], 1.0, 150)
    assert sea < DELTA_FLOOR, sea
    assert land > 10 * DELTA_FLOOR, land
