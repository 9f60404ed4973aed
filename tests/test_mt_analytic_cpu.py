"""The oracle against an analytic answer: the 1-D MT layered-earth check of
the reference's paper, on the reference's own serial example mesh
(serial/gen_mesh.f90: 51 air cells over 1000 ohm-m to 19 km, 10 ohm-m to
20 km and 100 ohm-m to the 50 km bottom), excited by the reference's MT sheet
sources (gen_rhs oper_mode 2 and 3, src/aphid.f90:590-619) at 0.01, 0.1 and
1 Hz, the frequencies of the paper's MT example.

This pin does not come from a restatement of the Fortran: the surface
impedance of the discrete solution (E_x / H_y and E_y / H_x at the surface)
is compared with the classical impedance recursion of a layered earth
(aphid_git_b200.mt.layered_impedance), whose bottom layer ends in the H = 0
wall that the mesh's homogeneous Neumann condition imposes at 50 km.  The
stated discretisation tolerance is 1.5% in apparent resistivity and 0.75
degrees in phase (measured: 0.02% / 0.06 deg at 1 Hz, 0.9% / 0.45 deg at
0.01 Hz, where the 1 km cells of the deep layers are coarsest against the
field's variation).  The sheet source and the Neumann sides make the
discrete solution exactly laterally uniform, so a 5 x 5 horizontal mesh has
the same impedance as the reference's 50 x 50 (checked: the impedance varies
by < 1e-9 across the surface).
"""
import numpy as np
import pytest

from aphid_git_b200 import model, mt
from oracle import oracle as O

FREQS = (0.01, 0.1, 1.0)
TOL_RHO, TOL_PHASE = 0.015, 0.75


def layers(zn, ks, sig):
    """interfaces and conductivities of the earth cells below node ks"""
    return zn[ks:], np.asarray(sig[0, 0, ks:], np.float64)


def oracle_impedance(f, nh=5, tol=1e-12):
    xn, yn, zn, sig, ks = model.serial_mt_model(nh)
    g = O.Grid(xn, yn, zn)
    w = 2 * np.pi * f
    k2 = O.gen_k2(g, model.sigma_hat("R", w, sig.ravel(order="F")), w)
    dg = O.gen_diag(g, k2)
    fields = []
    for mode in (2, 3):
        b = O.gen_rhs(g, mode)[0]
        r = O.qmr(g, k2, dg, b, tol, 20000)
        assert r["converged"]
        B, E = O.gen_fields(g, w, r["x"])
        fields.append([mt.surface_fields((nh, nh, len(zn)), ks, w, B, E, i, j)
                       for i in range(1, nh - 1) for j in range(1, nh - 1)])
    Z = np.array([mt.tensor(e1, h1, e2, h2) for (e1, h1), (e2, h2) in zip(*fields)])
    return Z, layers(zn, ks, sig)


@pytest.mark.parametrize("f", FREQS)
def test_oracle_surface_impedance_matches_layered_earth(f):
    Z, (depths, sig) = oracle_impedance(f)
    # laterally uniform: one impedance for every interior surface node
    assert np.max(np.abs(Z - Z[0])) < 1e-9 * np.abs(Z[0][0, 1])
    z = Z[0]
    za = mt.layered_impedance(f, depths, sig, bottom="wall")
    assert abs(z[0, 0]) < 1e-9 * abs(z[0, 1]) and abs(z[1, 1]) < 1e-9 * abs(z[0, 1])
    assert abs(z[1, 0] + z[0, 1]) < 1e-9 * abs(z[0, 1])   # Zyx = -Zxy in 1-D
    rho, ph = mt.apparent_resistivity(z[0, 1], f)
    rho_a, ph_a = mt.apparent_resistivity(za, f)
    assert abs(rho / rho_a - 1) < TOL_RHO, (f, rho, rho_a)
    assert abs(ph - ph_a) < TOL_PHASE, (f, ph, ph_a)


def test_layered_impedance_limits():
    """the recursion on its own: a uniform stack is a half-space (rho_a =
    1/sigma, 45 degrees without displacement currents), and a thin wall
    layer leaves a thick cover's impedance unchanged"""
    f = 0.3
    z = mt.layered_impedance(f, [0, 100, 900, 5000], [0.02] * 3, bottom="halfspace")
    w = 2 * np.pi * f
    k = np.sqrt(1j * w * model.MU0 * (0.02 + 1j * w * model.EPS0))
    assert abs(z - 1j * w * model.MU0 / k) < 1e-12 * abs(z)
    rho, ph = mt.apparent_resistivity(z, f)
    assert abs(rho - 50.0) < 1e-6 and abs(ph - 45.0) < 1e-6
    deep = mt.layered_impedance(f, [0, 2e5, 2e5 + 1], [0.02, 1.0], bottom="wall")
    assert abs(deep / z - 1) < 1e-6
