"""The VTK writers (the reference's dump_sigma, dump_fields, dump_a_phi,
src/aphid.f90:1731-2166) on CPU: Fortran e14.7 number form, header lines in
the reference's formats, and every array read back equal to what was
written within the 7 significant digits of e14.7.  Fields come from the
oracle's gen_fields on a small solved model."""
import numpy as np
import pytest

from aphid_git_b200 import model, vtk
from oracle import oracle as O


def test_fortran_e14_7():
    assert vtk.fortran_e(1234.5678) == " 0.1234568E+04"
    assert vtk.fortran_e(-0.000123456789) == "-0.1234568E-03"
    assert vtk.fortran_e(0.0) == " 0.0000000E+00"
    assert vtk.fortran_e(1.0) == " 0.1000000E+01"
    assert vtk.fortran_e(9.99999999) == " 0.1000000E+02"   # rounding carries into the exponent
    assert vtk.fortran_e(1e-120) == " 0.1000000-119"       # three-digit exponent drops the E
    for v in np.random.default_rng(1).standard_normal(200) * 10.0 ** np.random.default_rng(2).integers(-30, 30, 200):
        t = vtk.fortran_e(v)
        assert len(t) == 14 and abs(float(t) / v - 1) < 5e-7


@pytest.fixture(scope="module")
def solved(tmp_path_factory):
    rng = np.random.default_rng(4)
    dims = (9, 8, 10)
    xn, yn = model.graded_axis(dims[0] - 1, 100.0, 2), model.graded_axis(dims[1] - 1, 100.0, 2)
    zn = model.depth_axis(dims[2] - 1, 3, 100.0, 2)
    sig_re = (10.0 ** rng.uniform(-3, 0, tuple(d - 1 for d in dims))).astype(np.float32)
    g = O.Grid(xn, yn, zn)
    w = 2 * np.pi * 3.0
    sig = model.sigma_hat("R", w, sig_re.ravel(order="F"))
    k2 = O.gen_k2(g, sig, w)
    b = O.gen_rhs(g, 5, [("+X", 4, 4, 4)])[0]
    x = O.qmr(g, k2, O.gen_diag(g, k2), b, 1e-10, 3000)["x"]
    B, E = O.gen_fields(g, w, x)
    d = tmp_path_factory.mktemp("vtk")
    vtk.dump_sigma(str(d), xn, yn, zn, sig)
    vtk.dump_a_phi(str(d), xn, yn, zn, x)
    vtk.dump_fields(str(d), xn, yn, zn, w, B, E, k2)
    return d, (xn, yn, zn), sig, x, B, E, k2, w


def close(a, b):
    return np.allclose(a, b, rtol=6e-7, atol=1e-300 + 6e-7 * np.abs(b).max())


def test_sigma_vtk(solved):
    d, (xn, yn, zn), sig, *_ = solved
    lines = open(d / "sigma.vtk").read().splitlines()
    assert lines[:5] == ["# vtk DataFile Version 3.0", "vtk output", "ASCII", "DATASET RECTILINEAR_GRID",
                         "DIMENSIONS   9   8  10 "]
    assert lines[5] == "X_COORDINATES        9 float"
    assert "CELL_DATA            504" in lines
    dims, coords, data = vtk.read_vtk(d / "sigma.vtk")
    assert close(coords[2], zn)
    s = sig.reshape((8, 7, 9), order="F")
    assert close(data["sig_real"], s.real) and close(data["sig_imag"], s.imag)


def test_field_vtk(solved):
    d, (xn, yn, zn), sig, x, B, E, k2, w = solved
    nx, ny, nz = len(xn), len(yn), len(zn)
    nbx = nx * (ny - 1) * (nz - 1)
    _, _, data = vtk.read_vtk(d / "Bx.vtk")
    bx = B[:nbx].reshape((nx, ny - 1, nz - 1), order="F")
    assert close(data["Bx_real"], bx.real) and close(data["Bx_imag"], bx.imag)
    assert "POINT_DATA            640" in open(d / "Ex.vtk").read()
    assert "POINT_DATA      630" in open(d / "Ey.vtk").read()
    dims, coords, data = vtk.read_vtk(d / "Ez.vtk")
    assert dims == (nx, ny, nz - 1) and close(coords[2], 0.5 * (zn[1:] + zn[:-1]))
    oz = (nx - 1) * ny * nz + nx * (ny - 1) * nz
    ez = E[oz:].reshape((nx, ny, nz - 1), order="F")
    assert close(data["Ez_real"], ez.real)
    dims, coords, grid = vtk.read_vtk(d / "EM_grid.vtk")
    assert dims == (nx - 2, ny - 2, nz - 2)
    ex = E[:(nx - 1) * ny * nz].reshape((nx - 1, ny, nz), order="F")
    assert close(grid["Ex_grid_real"], (0.5 * (ex[:-1, 1:-1, 1:-1] + ex[1:, 1:-1, 1:-1])).real)
    k2x = k2[:(nx - 1) * ny * nz].reshape((nx - 1, ny, nz), order="F")
    jx = (ex[:-1, 1:-1, 1:-1] * k2x[:-1, 1:-1, 1:-1] + ex[1:, 1:-1, 1:-1] * k2x[1:, 1:-1, 1:-1]) / (2j * w * model.MU0)
    assert close(grid["Jx_grid_imag"], jx.imag)
    _, _, ap = vtk.read_vtk(d / "A_phi.vtk")
    ph = x[-nx * ny * nz:].reshape((nx, ny, nz), order="F")
    assert close(ap["phi_real"], ph[1:-1, 1:-1, 1:-1].real)
