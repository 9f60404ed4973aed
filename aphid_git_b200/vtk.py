"""ASCII VTK output of the reference's dump routines (src/aphid.f90:1731-2166).

The reference writes its results as legacy-VTK RECTILINEAR_GRID files:
  sigma.vtk     dump_sigma (src/aphid.f90:1803-1838): complex cell sigma-hat
  Bx.vtk ...    dump_fields (:1844-2031): the six field components on their
  Ez.vtk        staggered locations
  EM_grid.vtk   dump_fields (:2033-2165): E, J = k^2 E / (i omega mu0) and B
                interpolated onto the interior nodes (unweighted means)
  A_phi.vtk     dump_a_phi (:1731-1796): the potentials on the interior nodes.
                The reference writes them to unit 11 without opening a file
                (dump_sigma closed it), so they land in the compiler's default
                file for that unit; here they go to A_phi.vtk.

Numbers are written as Fortran's e14.7 edit descriptor prints them
(" 0.1234568E+04": sign, "0.", seven digits, a two-digit exponent), 1000 per
line with one blank after each, as the reference's `format(1000(e14.7,1x))`;
header lines follow its `(a,3(i3,1x))`, `(a,i8,a)` and `(a,i14,a)` formats.
Arrays are the reference's Fortran-ordered blocks (numpy arrays in Fortran
order, or flat in that order).
"""
import os

import numpy as np

from .model import MU0

_PER_LINE = 1000


def fortran_e(v):
    """one value in Fortran's e14.7 form"""
    v = float(v)
    if v == 0.0 or not np.isfinite(v):
        return " 0.0000000E+00" if v == 0.0 else ("%14s" % ("NaN" if v != v else ("Infinity" if v > 0 else "-Infinity")))
    s = "%.6E" % v                      # d.ddddddE+xx: 7 significant digits
    neg = s[0] == "-"
    body = s[1:] if neg else s
    mant, ex = body.split("E")
    e = int(ex) + 1                     # 0.ddddddd x 10^(e)
    digits = mant.replace(".", "")
    if abs(e) <= 99:
        tail = "E%+03d" % e
    else:
        tail = "%+04d" % e              # Fortran drops the E for three-digit exponents
    out = ("-" if neg else "") + "0." + digits + tail
    return out.rjust(14)


def _values(f, a):
    a = np.asarray(a, dtype=np.float64).ravel(order="F")
    for s in range(0, len(a), _PER_LINE):
        f.write("".join(fortran_e(v) + " " for v in a[s:s + _PER_LINE]) + "\n")


def _header(f, dims, coords):
    f.write("# vtk DataFile Version 3.0\n")
    f.write("vtk output\n")
    f.write("ASCII\n")
    f.write("DATASET RECTILINEAR_GRID\n")
    f.write("DIMENSIONS " + "".join("%3d " % d for d in dims) + "\n")
    for name, c in zip(("X", "Y", "Z"), coords):
        f.write("%s_COORDINATES %8d float\n" % (name, len(c)))
        _values(f, c)


def _scalar(f, name, a, kind="double"):
    f.write("SCALARS %s %s 1\n" % (name, kind))
    f.write("LOOKUP_TABLE default\n")
    _values(f, a)


def _mid(c):
    c = np.asarray(c, np.float64)
    return 0.5 * (c[:-1] + c[1:])


def dump_sigma(outdir, xn, yn, zn, sig):
    """sigma.vtk: the complex cell conductivity sigma-hat, (nx-1, ny-1, nz-1)."""
    nx, ny, nz = len(xn), len(yn), len(zn)
    sig = np.asarray(sig).reshape((nx - 1, ny - 1, nz - 1), order="F")
    with open(os.path.join(outdir, "sigma.vtk"), "w") as f:
        _header(f, (nx, ny, nz), (xn, yn, zn))
        f.write("CELL_DATA %14d\n" % ((nx - 1) * (ny - 1) * (nz - 1)))
        _scalar(f, "sig_real", sig.real, "float")
        _scalar(f, "sig_imag", sig.imag, "float")


def _blocks(nx, ny, nz, v):
    v = np.asarray(v)
    o = [0, (nx - 1) * ny * nz]
    o.append(o[1] + nx * (ny - 1) * nz)
    o.append(o[2] + nx * ny * (nz - 1))
    shapes = [(nx - 1, ny, nz), (nx, ny - 1, nz), (nx, ny, nz - 1), (nx, ny, nz)]
    return [v[o[q]:o[q] + int(np.prod(shapes[q]))].reshape(shapes[q], order="F") for q in range(len(o))]


def dump_a_phi(outdir, xn, yn, zn, sol):
    """A_phi.vtk: Ax, Ay, Az (means of the two edges through each node) and
    Phi on the interior nodes, from a solution vector [Ax|Ay|Az|Phi]."""
    nx, ny, nz = len(xn), len(yn), len(zn)
    ax, ay, az, ph = _blocks(nx, ny, nz, sol)
    i, j, k = slice(1, nx - 1), slice(1, ny - 1), slice(1, nz - 1)
    with open(os.path.join(outdir, "A_phi.vtk"), "w") as f:
        _header(f, (nx - 2, ny - 2, nz - 2), (xn[1:-1], yn[1:-1], zn[1:-1]))
        f.write("POINT_DATA %8d\n" % ((nx - 2) * (ny - 2) * (nz - 2)))
        a = 0.5 * (ax[0:nx - 2, j, k] + ax[1:nx - 1, j, k])
        _scalar(f, "Ax_real", a.real)
        _scalar(f, "Ax_imag", a.imag)
        a = 0.5 * (ay[i, 0:ny - 2, k] + ay[i, 1:ny - 1, k])
        _scalar(f, "Ay_real", a.real)
        _scalar(f, "Ay_imag", a.imag)
        a = 0.5 * (az[i, j, 0:nz - 2] + az[i, j, 1:nz - 1])
        _scalar(f, "Az_real", a.real)
        _scalar(f, "Az_imag", a.imag)
        _scalar(f, "phi_real", ph[i, j, k].real)
        _scalar(f, "phi_imag", ph[i, j, k].imag)


def dump_fields(outdir, xn, yn, zn, omega, B, E, k2):
    """Bx.vtk, By.vtk, Bz.vtk, Ex.vtk, Ey.vtk, Ez.vtk and EM_grid.vtk from the
    field arrays of gen_fields (B: [Bx|By|Bz] on faces, E: [Ex|Ey|Ez] on
    edges) and the k^2 grids [x|y|z|p] (for J on the nodes).  EM_grid's
    By_grid keeps the reference's expression, which takes the face
    By(i, j, k-1) twice and omits By(i-1, j, k) (src/aphid.f90:2140-2149)."""
    nx, ny, nz = len(xn), len(yn), len(zn)
    B, E = np.asarray(B), np.asarray(E)
    nbx, nby = nx * (ny - 1) * (nz - 1), (nx - 1) * ny * (nz - 1)
    bx = B[:nbx].reshape((nx, ny - 1, nz - 1), order="F")
    by = B[nbx:nbx + nby].reshape((nx - 1, ny, nz - 1), order="F")
    bz = B[nbx + nby:].reshape((nx - 1, ny - 1, nz), order="F")
    ex, ey, ez = _blocks(nx, ny, nz, np.concatenate([E, np.zeros(nx * ny * nz, E.dtype)]))[:3]
    k2x, k2y, k2z, _ = _blocks(nx, ny, nz, k2)
    xm, ym, zm = _mid(xn), _mid(yn), _mid(zn)
    comps = [("Bx", bx, (xn, ym, zm)), ("By", by, (xm, yn, zm)), ("Bz", bz, (xm, ym, zn)),
             ("Ex", ex, (xm, yn, zn)), ("Ey", ey, (xn, ym, zn)), ("Ez", ez, (xn, yn, zm))]
    for name, a, coords in comps:
        with open(os.path.join(outdir, name + ".vtk"), "w") as f:
            _header(f, a.shape, coords)
            # the reference's formats: i14 for Bx, By, Bz and Ex, i8 for Ey and Ez
            f.write(("POINT_DATA %8d\n" if name in ("Ey", "Ez") else "POINT_DATA %14d\n") % a.size)
            _scalar(f, name + "_real", a.real)
            _scalar(f, name + "_imag", a.imag)
    I, J, K = slice(1, nx - 1), slice(1, ny - 1), slice(1, nz - 1)
    lo_i, lo_j, lo_k = slice(0, nx - 2), slice(0, ny - 2), slice(0, nz - 2)
    w = 2.0 * 1j * omega * MU0
    grid = {
        "Ex_grid": (ex[lo_i, J, K] + ex[I, J, K]) / 2.0,
        "Ey_grid": (ey[I, lo_j, K] + ey[I, J, K]) / 2.0,
        "Ez_grid": (ez[I, J, lo_k] + ez[I, J, K]) / 2.0,
        "Jx_grid": (ex[lo_i, J, K] * k2x[lo_i, J, K] + ex[I, J, K] * k2x[I, J, K]) / w,
        "Jy_grid": (ey[I, lo_j, K] * k2y[I, lo_j, K] + ey[I, J, K] * k2y[I, J, K]) / w,
        "Jz_grid": (ez[I, J, K] * k2z[I, J, K] + ez[I, J, lo_k] * k2z[I, J, lo_k]) / w,
        "Bx_grid": (bx[I, lo_j, lo_k] + bx[I, J, lo_k] + bx[I, lo_j, K] + bx[I, J, K]) / 4.0,
        "By_grid": (by[lo_i, J, lo_k] + by[I, J, lo_k] + by[I, J, lo_k] + by[I, J, K]) / 4.0,
        "Bz_grid": (bz[lo_i, lo_j, K] + bz[lo_i, J, K] + bz[I, lo_j, K] + bz[I, J, K]) / 4.0,
    }
    with open(os.path.join(outdir, "EM_grid.vtk"), "w") as f:
        _header(f, (nx - 2, ny - 2, nz - 2), (xn[1:-1], yn[1:-1], zn[1:-1]))
        f.write("POINT_DATA %8d\n" % ((nx - 2) * (ny - 2) * (nz - 2)))
        for name, a in grid.items():
            _scalar(f, name + "_real", a.real)
            _scalar(f, name + "_imag", a.imag)


def read_vtk(path):
    """Parse a file written above: returns (dims, coords, {name: array}) with
    the arrays in Fortran order, shaped by DIMENSIONS (or cell counts)."""
    with open(path) as f:
        lines = f.read().splitlines()
    dims = tuple(int(t) for t in lines[4].split()[1:4])
    pos, coords, data = 5, [], {}

    def take(n):
        nonlocal pos
        vals = []
        while len(vals) < n:
            vals += [float(t) for t in lines[pos].split()]
            pos += 1
        return np.array(vals)

    for _ in range(3):
        n = int(lines[pos].split()[1])
        pos += 1
        coords.append(take(n))
    count = int(lines[pos].split()[1])
    cell = lines[pos].startswith("CELL_DATA")
    pos += 1
    shape = tuple(d - 1 for d in dims) if cell else dims
    while pos < len(lines) and lines[pos].startswith("SCALARS"):
        name = lines[pos].split()[1]
        pos += 2
        data[name] = take(count).reshape(shape, order="F")
    return dims, coords, data
