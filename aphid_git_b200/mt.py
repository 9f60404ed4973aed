"""Magnetotelluric post-processing: the impedance tensor from the two MT
source polarisations, and the analytic impedance of a 1-D layered earth.

The reference leaves impedance "as a post-processing exercise"
(man/aphid.1:159-160); its MT sources are the sheet currents of gen_rhs
oper_mode 2 (x-polarised) and 3 (y-polarised) (src/aphid.f90:590-619).  With
E and H of both polarisations at a site, Z solves

    [Ex1 Ex2]   [Zxx Zxy] [Hx1 Hx2]
    [Ey1 Ey2] = [Zyx Zyy] [Hy1 Hy2],

and the apparent resistivity and phase are rho_a = |Z|^2 / (omega mu0),
phi = arg Z.  The fields follow the reference's conventions: time factor
exp(i omega t) (E = -i omega (A - grad Phi), src/aphid.f90:2225-2250) and z
positive downwards, so a wave travelling down into a half-space of
conductivity sigma has Zxy = i omega mu0 / k with k = sqrt(i omega mu0 sigma).

layered_impedance is the classical recursion of a stack of uniform layers
(Wait, 1954; e.g. Ward & Hohmann, 1988, eq. 4.183), written here from the
formula: for layer j with k_j = sqrt(i omega mu0 sigma-hat_j) and intrinsic
impedance Z0_j = i omega mu0 / k_j, the impedance at its top is
Z0_j (Z_below + Z0_j tanh(k_j h_j)) / (Z0_j + Z_below tanh(k_j h_j)).  The
bottom is either a half-space (Z_below of the last layer = its Z0) or, as
in a mesh whose last node carries the reference's homogeneous Neumann
condition (dA/dz = 0, so H = 0 there), a wall with Z_below = infinity,
giving Z0 coth(k h) for the last layer.
"""
import numpy as np

from .model import EPS0, MU0


def layered_impedance(freq, depths, sigma, bottom="halfspace", eps_rel=None):
    """Surface impedance E_x / H_y of a 1-D layered earth.

    depths: the N+1 interface depths (m, increasing), the first the surface;
    sigma: N layer conductivities (S/m); the last layer ends at depths[-1]
    ("wall": H = 0 there) or continues down ("halfspace").  eps_rel
    (optional) adds displacement currents, sigma-hat = sigma + i omega eps0
    eps_r, as the reference's conductivity model R (eps_r = 1) does."""
    w = 2.0 * np.pi * float(freq)
    h = np.diff(np.asarray(depths, np.float64))
    sig = np.asarray(sigma, np.float64)
    er = np.ones_like(sig) if eps_rel is None else np.asarray(eps_rel, np.float64)
    if len(h) != len(sig):
        raise ValueError("need one conductivity per layer")
    k = np.sqrt(1j * w * MU0 * (sig + 1j * w * EPS0 * er))
    z0 = 1j * w * MU0 / k
    if bottom == "wall":
        z = z0[-1] / np.tanh(k[-1] * h[-1])
    elif bottom == "halfspace":
        z = z0[-1]
    else:
        raise ValueError("bottom must be 'wall' or 'halfspace'")
    for j in range(len(h) - 2, -1, -1):
        t = np.tanh(k[j] * h[j])
        z = z0[j] * (z + z0[j] * t) / (z0[j] + z * t)
    return z


def tensor(E1, H1, E2, H2):
    """Impedance tensors from the horizontal fields of the two polarisations
    (..., 2) arrays of (x, y) components: returns (..., 2, 2)."""
    E = np.stack([np.asarray(E1)[..., :2], np.asarray(E2)[..., :2]], axis=-1)
    H = np.stack([np.asarray(H1)[..., :2], np.asarray(H2)[..., :2]], axis=-1)
    return E @ np.linalg.inv(H)


def apparent_resistivity(Z, freq):
    """rho_a = |Z|^2 / (omega mu0) in ohm-m, phase in degrees"""
    w = 2.0 * np.pi * float(freq)
    return np.abs(Z) ** 2 / (w * MU0), np.degrees(np.angle(Z))


def surface_fields(dims, zn_surface_index, omega, B, E, i, j):
    """E and H at surface node (i, j, ks) (0-based) from full field arrays
    (gen_fields layout): E on the node from the mean of the two edges along
    x and y, H from the faces of the air cell just above the surface, where
    H is uniform in z (air carries no current), averaged over the two faces
    on either side of the node.  Returns (E (3,), H (3,))."""
    nx, ny, nz = dims
    ks = zn_surface_index
    oy = (nx - 1) * ny * nz
    oz = oy + nx * (ny - 1) * nz
    ex = E[:oy].reshape((nx - 1, ny, nz), order="F")
    ey = E[oy:oz].reshape((nx, ny - 1, nz), order="F")
    nbx, nby = nx * (ny - 1) * (nz - 1), (nx - 1) * ny * (nz - 1)
    bx = B[:nbx].reshape((nx, ny - 1, nz - 1), order="F")
    by = B[nbx:nbx + nby].reshape((nx - 1, ny, nz - 1), order="F")
    e = np.array([0.5 * (ex[i - 1, j, ks] + ex[i, j, ks]), 0.5 * (ey[i, j - 1, ks] + ey[i, j, ks]), 0.0])
    h = np.array([0.5 * (bx[i, j - 1, ks - 1] + bx[i, j, ks - 1]),
                  0.5 * (by[i - 1, j, ks - 1] + by[i, j, ks - 1]), 0.0]) / MU0
    return e, h
