"""ctypes view of the CPU oracle (oracle/aphid_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, always as the checker or the timed CPU
baseline, never by the product package.

Parity status: parity unpinned against a reference binary (the reference is
Fortran 90 and no Fortran compiler exists here).  The restatement is pinned
by tests/golden (independent NumPy/SciPy assembly), structural identities,
a sparse direct solve and the 1-D MT analytic solution.

All vectors are numpy complex128 arrays in the reference's unknown order
[Ax(nx-1,ny,nz) | Ay(nx,ny-1,nz) | Az(nx,ny,nz-1) | Phi(nx,ny,nz)], each
block Fortran-ordered (i fastest).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libaphid_oracle.so")
_lib = None


def build(force=False):
    """Compile the oracle with oracle/Makefile (gcc)."""
    if force or not os.path.exists(_SO):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_SO)
        dp = C.POINTER(C.c_double)
        vp = C.c_void_p
        L.orc_spacings.argtypes = [C.c_int, vp, vp, vp]
        L.orc_sigma_hat.argtypes = [C.c_char, C.c_size_t, C.c_double, vp, vp, vp, vp, vp, vp]
        L.orc_sigma_hat.restype = C.c_int
        L.orc_gen_k2.argtypes = [C.c_int] * 3 + [vp] * 3 + [vp, C.c_double, vp]
        L.orc_gen_diag.argtypes = [C.c_int] * 3 + [vp] * 5
        L.orc_inprod.argtypes = [C.c_int] * 3 + [vp] * 9
        L.orc_gen_rhs.argtypes = [C.c_int] * 4 + [vp] * 6 + [C.c_int, C.c_char_p, vp, vp, vp]
        L.orc_gen_rhs.restype = C.c_int
        L.orc_qmr.argtypes = ([C.c_int] * 3 + [vp] * 6 + [vp, vp, vp, vp, C.c_double, C.c_int,
                              C.c_int, vp, C.c_int, dp, dp, C.POINTER(C.c_int), dp])
        L.orc_qmr.restype = C.c_int
        L.orc_gen_fields.argtypes = [C.c_int] * 3 + [vp] * 3 + [C.c_double, vp, vp, vp]
        L.orc_nunk.argtypes = [C.c_int] * 3
        L.orc_nunk.restype = C.c_size_t
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def nunk(nx, ny, nz):
    return (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1) + nx * ny * nz


class Grid:
    """Node coordinates and the reference's spacing arrays dx(0:n), dxc(1:n)."""

    def __init__(self, xn, yn, zn):
        self.xn, self.yn, self.zn = _f64(xn), _f64(yn), _f64(zn)
        self.nx, self.ny, self.nz = len(self.xn), len(self.yn), len(self.zn)
        self.dx, self.dxc = spacings(self.xn)
        self.dy, self.dyc = spacings(self.yn)
        self.dz, self.dzc = spacings(self.zn)
        self.n = nunk(self.nx, self.ny, self.nz)

    @property
    def dims(self):
        return self.nx, self.ny, self.nz


def spacings(xn):
    xn = _f64(xn)
    n = len(xn)
    d = np.zeros(n + 1)
    dc = np.zeros(n)
    lib().orc_spacings(n, _p(xn), _p(d), _p(dc))
    return d, dc


def sigma_hat(mode, omega, sig_re=None, eps_rel=None, eta=None, tau=None, cee=None):
    """Cell sigma-hat (complex128, Fortran order) from real(4) cell arrays."""
    arrs = [sig_re, eps_rel, eta, tau, cee]
    ref = next(a for a in arrs if a is not None)
    ncell = np.asarray(ref).size
    f32 = [np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel(order="F"))
           if a is not None else np.zeros(ncell, np.float32) for a in arrs]
    out = np.zeros(ncell, np.complex128)
    rc = lib().orc_sigma_hat(mode.encode(), ncell, omega, *[_p(a) for a in f32], _p(out))
    if rc != 0:
        raise ValueError("bad conductivity mode %r" % mode)
    return out


def gen_k2(g, sig, omega):
    sig = _c128(sig)
    out = np.zeros(g.n, np.complex128)
    lib().orc_gen_k2(g.nx, g.ny, g.nz, _p(g.dx), _p(g.dy), _p(g.dz), _p(sig), omega, _p(out))
    return out


def gen_diag(g, k2):
    k2 = _c128(k2)
    out = np.zeros(g.n, np.complex128)
    lib().orc_gen_diag(g.nx, g.ny, g.nz, _p(g.dx), _p(g.dy), _p(g.dz), _p(k2), _p(out))
    return out


def inprod(g, k2, x):
    k2, x = _c128(k2), _c128(x)
    y = np.zeros(g.n, np.complex128)
    lib().orc_inprod(g.nx, g.ny, g.nz, _p(g.dx), _p(g.dy), _p(g.dz), _p(g.dxc), _p(g.dyc),
                     _p(g.dzc), _p(k2), _p(x), _p(y))
    return y


def gen_rhs(g, mode, dipoles=()):
    """dipoles: iterable of (dir, i, j, k) with dir in +X,-X,+Y,-Y,+Z,-Z."""
    dipoles = list(dipoles)
    dirs = "".join(d[0][:2].ljust(2) for d in dipoles).encode() or b"  "
    ijk = np.array([[d[1], d[2], d[3]] for d in dipoles] or [[0, 0, 0]], dtype=np.int32)
    out = np.zeros(g.n, np.complex128)
    nsk = C.c_int(0)
    rc = lib().orc_gen_rhs(mode, g.nx, g.ny, g.nz, _p(g.xn), _p(g.yn), _p(g.zn), _p(g.dx),
                           _p(g.dy), _p(g.dz), len(dipoles), dirs, _p(ijk), _p(out),
                           C.byref(nsk))
    if rc != 0:
        raise ValueError("gen_rhs failed for mode %d" % mode)
    return out, nsk.value


def qmr(g, k2, diag, b, target, max_it, x0=None, nthreads=1):
    """Returns dict(x, iters, hist, rnorm, rhsnorm, converged, seconds)."""
    k2, diag = _c128(k2), _c128(diag)
    x = _c128(b).copy()
    hist = np.zeros(max(1, max_it) + 1)
    rn, bn, sec = C.c_double(), C.c_double(), C.c_double()
    conv = C.c_int()
    x0p = _p(_c128(x0)) if x0 is not None else None
    it = lib().orc_qmr(g.nx, g.ny, g.nz, _p(g.dx), _p(g.dy), _p(g.dz), _p(g.dxc), _p(g.dyc),
                       _p(g.dzc), _p(k2), _p(diag), _p(x), x0p, target, max_it, nthreads,
                       _p(hist), len(hist), C.byref(rn), C.byref(bn), C.byref(conv),
                       C.byref(sec))
    nh = min(it if conv.value else max(1, max_it), len(hist))
    return dict(x=x, iters=it, hist=hist[:nh], rnorm=rn.value, rhsnorm=bn.value,
                converged=bool(conv.value), seconds=sec.value)


def gen_fields(g, omega, sol):
    sol = _c128(sol)
    nb = g.nx * (g.ny - 1) * (g.nz - 1) + (g.nx - 1) * g.ny * (g.nz - 1) + \
        (g.nx - 1) * (g.ny - 1) * g.nz
    ne = g.n - g.nx * g.ny * g.nz
    B = np.zeros(nb, np.complex128)
    E = np.zeros(ne, np.complex128)
    lib().orc_gen_fields(g.nx, g.ny, g.nz, _p(g.dx), _p(g.dy), _p(g.dz), omega, _p(sol),
                         _p(B), _p(E))
    return B, E
