"""Generate golden fixtures for the APhiD operator and QMR solve.

The reference (Fortran 90 + OpenMP + MPI) cannot be compiled on this machine
or on the GPU machine and ships no tests or fixtures, so these fixtures come
from an INDEPENDENT restatement: a vectorised NumPy/SciPy assembly of the
sparse operator K written from the reference's formulas (src/aphid.f90), a
NumPy QMR (src/aphid_qmr.f90:5-434) on that sparse matrix, and SciPy's sparse
direct solve.  The C oracle (oracle/aphid_oracle.c) is a loop-by-loop
restatement; agreement between the two pins indexing and operation order.

Run:  python tests/golden/make_golden.py      (writes tests/golden/*.npz)
"""
import os
import sys

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

MU0 = np.pi * 4e-7
EPS0 = 8.8541878176e-12
HERE = os.path.dirname(os.path.abspath(__file__))


# ---------------------------------------------------------------- geometry
def ref_spacing(xn):
    """dx(0:n) and dxc(1:n) as numpy arrays d[0..n], dc[0..n-1]."""
    h = np.diff(xn)
    d = np.concatenate([[h[0]], h, [h[-1]]])
    dc = np.empty(len(xn))
    dc[1:-1] = 0.5 * (h[:-1] + h[1:])
    dc[0], dc[-1] = dc[1], dc[-2]
    return d, dc


def sigma_hat(mode, omega, sig_re, eps_rel, eta, tau, cee):
    s = sig_re.astype(np.float64)
    if mode == "R":
        return s + 1j * omega * EPS0
    if mode == "C":
        return s + 1j * omega * EPS0 * eps_rel.astype(np.float64)
    if mode == "D":
        z = (1j * omega * tau.astype(np.float64)) ** cee.astype(np.float64)
        return s * (1.0 - eta.astype(np.float64) / (1.0 + z))
    if mode == "I":
        return 1j * omega * EPS0 * eps_rel.astype(np.float64)
    raise ValueError(mode)


def clamp_idx(n):
    return np.clip(np.arange(n), 1, n - 2)


def wavenumbers(xn, yn, zn, sig, omega):
    """k2 on x/y/z edges and nodes (src/aphid.f90:1289-1535): area / volume
    weighted cell averages on the interior, boundary values copied from the
    nearest interior point (every copy there reduces to index clamping)."""
    hx, hy, hz = np.diff(xn), np.diff(yn), np.diff(zn)
    nx, ny, nz = len(xn), len(yn), len(zn)
    fac = 1j * omega * MU0

    def full(shape):
        return np.zeros(shape, complex)

    # x-edges: average over the 4 cells around the edge in (y,z)
    kx = full((nx - 1, ny, nz))
    J, K = np.meshgrid(np.arange(1, ny - 1), np.arange(1, nz - 1), indexing="ij")
    wy0, wy1, wz0, wz1 = hy[J - 1], hy[J], hz[K - 1], hz[K]
    num = (sig[:, J - 1, K - 1] * (wy0 * wz0) + sig[:, J, K - 1] * (wy1 * wz0)
           + sig[:, J, K] * (wy1 * wz1) + sig[:, J - 1, K] * (wy0 * wz1))
    kx[:, 1:-1, 1:-1] = num / ((wy0 + wy1) * (wz0 + wz1))
    kx = kx[:, clamp_idx(ny)][:, :, clamp_idx(nz)]

    ky = full((nx, ny - 1, nz))
    I, K = np.meshgrid(np.arange(1, nx - 1), np.arange(1, nz - 1), indexing="ij")
    wx0, wx1, wz0, wz1 = hx[I - 1], hx[I], hz[K - 1], hz[K]
    s = sig.transpose(0, 2, 1)  # (cx, cz, cy)
    num = (s[I - 1, K - 1] * (wx0 * wz0)[..., None] + s[I, K - 1] * (wx1 * wz0)[..., None]
           + s[I, K] * (wx1 * wz1)[..., None] + s[I - 1, K] * (wx0 * wz1)[..., None])
    val = num / ((wx0 + wx1) * (wz0 + wz1))[..., None]  # (nx-2, nz-2, ny-1)
    ky[1:-1, :, 1:-1] = val.transpose(0, 2, 1)
    ky = ky[clamp_idx(nx)][:, :, clamp_idx(nz)]

    kz = full((nx, ny, nz - 1))
    I, J = np.meshgrid(np.arange(1, nx - 1), np.arange(1, ny - 1), indexing="ij")
    wx0, wx1, wy0, wy1 = hx[I - 1], hx[I], hy[J - 1], hy[J]
    num = (sig[I - 1, J - 1] * (wx0 * wy0)[..., None] + sig[I, J - 1] * (wx1 * wy0)[..., None]
           + sig[I, J] * (wx1 * wy1)[..., None] + sig[I - 1, J] * (wx0 * wy1)[..., None])
    kz[1:-1, 1:-1, :] = num / ((wx0 + wx1) * (wy0 + wy1))[..., None]
    kz = kz[clamp_idx(nx)][:, clamp_idx(ny)]

    kp = full((nx, ny, nz))
    I, J, K = np.meshgrid(np.arange(1, nx - 1), np.arange(1, ny - 1), np.arange(1, nz - 1),
                          indexing="ij")
    acc = 0
    for di in (0, 1):
        for dj in (0, 1):
            for dk in (0, 1):
                w = hx[I - 1 + di] * hy[J - 1 + dj] * hz[K - 1 + dk]
                acc = acc + sig[I - 1 + di, J - 1 + dj, K - 1 + dk] * w
    kp[1:-1, 1:-1, 1:-1] = acc / ((hx[I - 1] + hx[I]) * (hy[J - 1] + hy[J]) * (hz[K - 1] + hz[K]))
    kp = kp[clamp_idx(nx)][:, clamp_idx(ny)][:, :, clamp_idx(nz)]
    return kx * fac, ky * fac, kz * fac, kp * fac


# ------------------------------------------------------------- the operator
class Blocks:
    def __init__(self, nx, ny, nz):
        self.shapes = [(nx - 1, ny, nz), (nx, ny - 1, nz), (nx, ny, nz - 1), (nx, ny, nz)]
        sizes = [int(np.prod(s)) for s in self.shapes]
        self.off = np.concatenate([[0], np.cumsum(sizes)])
        self.n = int(self.off[-1])

    def gid(self, b, i, j, k):
        n1, n2, _ = self.shapes[b]
        return self.off[b] + i + n1 * (j + n2 * k)

    def split(self, v):
        return [v[self.off[b]:self.off[b + 1]].reshape(self.shapes[b], order="F")
                for b in range(4)]

    def join(self, blocks):
        return np.concatenate([np.asarray(x).ravel(order="F") for x in blocks])


def lap_coefs(d, dc, n):
    """1-D Neumann Laplacian couplings along one axis.
    edge-type (component along the axis), 0-based edge e in 0..n-2:
        up[e] = -1/(dc[e+1] d[e+1]) unless e == n-2;  dn[e] = -1/(dc[e] d[e+1]) unless e == 0
    node-type (transverse components and Phi), 0-based node m in 0..n-1:
        up[m] = -1/(d[m+1] dc[m]) unless m == n-1;  dn[m] = -1/(d[m] dc[m]) unless m == 0
    (d is dx(0:n) and dc is dxc(1:n), both 0-based numpy arrays)."""
    e = np.arange(n - 1)
    eu = np.where(e == n - 2, 0.0, -1.0 / dc[e + 1] / d[e + 1])
    ed = np.where(e == 0, 0.0, -1.0 / dc[e] / d[e + 1])
    m = np.arange(n)
    nu = np.where(m == n - 1, 0.0, -1.0 / d[m + 1] / dc[m])
    nd = np.where(m == 0, 0.0, -1.0 / d[m] / dc[m])
    return eu, ed, nu, nd


def assemble(xn, yn, zn, k2):
    """Sparse K (complex128) from the formulas of inprod_x/y/z/p
    (src/aphid.f90:803-1282).  Edge rows: 7-point Neumann Laplacian plus k2
    on the diagonal, plus the gradient of Phi weighted by (k2_node - k2_edge);
    rows scaled by the dual volume.  Node rows (interior only): the
    k2-weighted Laplacian with k2^2 on the diagonal, plus the divergence
    coupling (k2_edge - k2_node) to the six incident edges."""
    nx, ny, nz = len(xn), len(yn), len(zn)
    B = Blocks(nx, ny, nz)
    axes = [(d, dc, lap_coefs(d, dc, n)) for (d, dc), n in
            zip((ref_spacing(xn), ref_spacing(yn), ref_spacing(zn)), (nx, ny, nz))]
    kx, ky, kz, kp = B.split(k2)
    kedge = [kx, ky, kz]
    rows, cols, vals = [], [], []

    def add(r, c, v):
        r, c, v = np.broadcast_arrays(r, c, v)
        rows.append(r.ravel()); cols.append(c.ravel()); vals.append(v.ravel())

    for b in range(3):
        shp = B.shapes[b]
        idx = np.meshgrid(*[np.arange(s) for s in shp], indexing="ij")
        row = B.gid(b, *idx)
        vol = np.ones(shp)
        for a in range(3):
            d, dc, _ = axes[a]
            vol = vol * (d[idx[a] + 1] if a == b else dc[idx[a]])
        diag = kedge[b].copy()
        for a in range(3):
            d, dc, (eu, ed, nu, nd) = axes[a]
            m = idx[a]
            up, dn = (eu[m], ed[m]) if a == b else (nu[m], nd[m])
            diag = diag - up - dn
            iu = list(idx); iu[a] = np.minimum(m + 1, shp[a] - 1)
            idn = list(idx); idn[a] = np.maximum(m - 1, 0)
            add(row, B.gid(b, *iu), up * vol)
            add(row, B.gid(b, *idn), dn * vol)
        add(row, row, diag * vol)
        ip = list(idx); ip[b] = idx[b] + 1
        g = vol / axes[b][0][idx[b] + 1]
        add(row, B.gid(3, *ip), (kp[tuple(ip)] - kedge[b]) * g)
        add(row, B.gid(3, *idx), -(kp[tuple(idx)] - kedge[b]) * g)

    I, J, Kk = np.meshgrid(np.arange(1, nx - 1), np.arange(1, ny - 1), np.arange(1, nz - 1),
                           indexing="ij")
    idx = [I, J, Kk]
    row = B.gid(3, I, J, Kk)
    vol = axes[0][1][I] * axes[1][1][J] * axes[2][1][Kk]
    s1 = kp[I, J, Kk]
    diag = s1 * s1
    for a in range(3):
        d, dc, (eu, ed, nu, nd) = axes[a]
        m = idx[a]
        ilo = list(idx); ilo[a] = m - 1
        s_hi, s_lo = kedge[a][tuple(idx)], kedge[a][tuple(ilo)]
        c_up, c_dn = nu[m] * s_hi, nd[m] * s_lo
        diag = diag - c_up - c_dn
        nb_hi = list(idx); nb_hi[a] = m + 1
        add(row, B.gid(3, *nb_hi), c_up * vol)
        add(row, B.gid(3, *ilo), c_dn * vol)
        add(row, B.gid(a, *idx), (s_hi - s1) / dc[m] * vol)
        add(row, B.gid(a, *ilo), -(s_lo - s1) / dc[m] * vol)
    add(row, row, diag * vol)
    K = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(B.n, B.n)).tocsr()
    K.sum_duplicates()
    return K


def jacobi_diag(xn, yn, zn, k2):
    """gen_diag (src/aphid.f90:1542-1725): like the true diagonal but with
    0.5*(d(k)+d(k-1)) in place of dxc, and 1 on the boundary nodes."""
    nx, ny, nz = len(xn), len(yn), len(zn)
    B = Blocks(nx, ny, nz)
    d3 = [ref_spacing(xn)[0], ref_spacing(yn)[0], ref_spacing(zn)[0]]
    n3 = [nx, ny, nz]
    kx, ky, kz, kp = B.split(k2)
    out = [np.ones(s, complex) for s in B.shapes]
    for b in range(3):
        shp = B.shapes[b]
        idx = np.meshgrid(*[np.arange(s) for s in shp], indexing="ij")
        vol = np.ones(shp)
        acc = np.zeros(shp)
        for a in range(3):
            d, n, m = d3[a], n3[a], idx[a]
            if a == b:  # edge along a: d(i) with half-sums d(i)+d(i+1), d(i)+d(i-1)
                dcp = 0.5 * (d[m + 1] + d[m + 2])
                dcm = 0.5 * (d[m + 1] + d[m])
                up = np.where(m == n - 2, 0.0, -1.0 / dcp / d[m + 1])
                dn = np.where(m == 0, 0.0, -1.0 / dcm / d[m + 1])
                vol = vol * d[m + 1]
            else:
                dcm = 0.5 * (d[m + 1] + d[m])
                up = np.where(m == n - 1, 0.0, -1.0 / d[m + 1] / dcm)
                dn = np.where(m == 0, 0.0, -1.0 / d[m] / dcm)
                vol = vol * dcm
            acc = acc + up + dn
        out[b] = (-acc + [kx, ky, kz][b]) * vol
    I, J, K = np.meshgrid(np.arange(1, nx - 1), np.arange(1, ny - 1), np.arange(1, nz - 1),
                          indexing="ij")
    idx = [I, J, K]
    vol = 1.0
    acc = 0
    ke = [kx, ky, kz]
    for a in range(3):
        d, m = d3[a], idx[a]
        dcm = 0.5 * (d[m + 1] + d[m])
        vol = vol * dcm
        lo = list(idx); lo[a] = m - 1
        acc = acc + (-ke[a][tuple(idx)] / d[m + 1] / dcm) + (-ke[a][tuple(lo)] / d[m] / dcm)
    s1 = kp[I, J, K]
    out[3][1:-1, 1:-1, 1:-1] = (-acc + s1 * s1) * vol
    return B.join(out)


def rhs_mode5(xn, yn, zn, dipoles):
    nx, ny, nz = len(xn), len(yn), len(zn)
    B = Blocks(nx, ny, nz)
    d3 = [ref_spacing(xn)[0], ref_spacing(yn)[0], ref_spacing(zn)[0]]
    n3 = [nx, ny, nz]
    v = np.zeros(B.n, complex)
    skipped = 0
    for dr, i, j, k in dipoles:
        if len(dr) != 2 or dr[0] not in "+-" or dr[1] not in "XYZ":
            skipped += 1
            continue
        a = "XYZ".index(dr[1])
        tail = [i, j, k]
        if dr[0] == "-":          # "-X i j k" is the +X dipole whose tail is i-1
            tail[a] -= 1
        head = list(tail); head[a] += 1
        lim = [n for n in n3]
        lim[a] -= 1               # edge index range along the dipole axis
        if any(t < 1 or t > l for t, l in zip(tail, lim)):
            skipped += 1
            continue
        sgn = 1.0 if dr[0] == "+" else -1.0
        t0 = [t - 1 for t in tail]
        h0 = [t - 1 for t in head]
        v[B.gid(a, *t0)] += sgn * MU0 * d3[a][tail[a]]
        v[B.gid(3, *t0)] += sgn * MU0
        v[B.gid(3, *h0)] -= sgn * MU0
    return v, skipped


def qmr_np(K, diag, b, target, max_it):
    """Freund-Nachtigal coupled two-term QMR with Jacobi preconditioning as
    in src/aphid_qmr.f90:5-434, on a SciPy matrix.  Returns x, iters, hist."""
    inv = 1.0 / diag
    bn = np.sqrt(np.vdot(b, b).real)
    x = np.zeros_like(b)
    r = b - K @ x
    vt = r.copy()
    rho = np.sqrt(np.vdot(r, r).real)
    v = vt / rho
    p = np.zeros_like(b); d = np.zeros_like(b); s = np.zeros_like(b)
    c, eps, theta, eta = 1.0, 1.0 + 0j, 0.0, -1.0 + 0j
    it, hist = 1, []
    while True:
        cm, rhon, thm = c, rho, theta
        t = v * inv
        dl = np.sum(v * t)
        k1 = rhon * dl / eps
        p = t - p * k1
        q = K @ p
        eps = np.sum(p * q)
        beta = eps / dl
        vt = q - v * beta
        rho = np.sqrt(np.vdot(vt, vt).real)
        theta = rho * rho / cm / (beta.real ** 2 + beta.imag ** 2)
        c = 1.0 / (1.0 + theta)
        eta = -eta * rhon * c / (beta * cm)
        kk = thm * c
        d = p * eta + d * kk
        x = x + d
        s = q * eta + s * kk
        r = r - s
        v = vt / rho
        rn = np.sqrt(np.vdot(r, r).real)
        hist.append(rn)
        conv = rn < target * bn
        if not conv and it <= max_it:
            it += 1
        if conv or it > max_it:
            break
    return x, it, np.array(hist), conv


def fields(xn, yn, zn, omega, sol):
    nx, ny, nz = len(xn), len(yn), len(zn)
    B = Blocks(nx, ny, nz)
    ax, ay, az, ph = B.split(sol)
    dx = ref_spacing(xn)[0][1:nx][:, None, None]
    dy = ref_spacing(yn)[0][1:ny][None, :, None]
    dz = ref_spacing(zn)[0][1:nz][None, None, :]
    bx = (az[:, 1:, :] - az[:, :-1, :]) / dy - (ay[:, :, 1:] - ay[:, :, :-1]) / dz
    by = (ax[:, :, 1:] - ax[:, :, :-1]) / dz - (az[1:, :, :] - az[:-1, :, :]) / dx
    bz = (ay[1:, :, :] - ay[:-1, :, :]) / dx - (ax[:, 1:, :] - ax[:, :-1, :]) / dy
    ex = -1j * omega * (ax - (ph[1:] - ph[:-1]) / dx)
    ey = -1j * omega * (ay - (ph[:, 1:] - ph[:, :-1]) / dy)
    ez = -1j * omega * (az - (ph[:, :, 1:] - ph[:, :, :-1]) / dz)
    return B.join([bx, by, bz]), B.join([ex, ey, ez])


# ------------------------------------------------------------------ cases
def graded(n, core, rng):
    h = core * (1.0 + 0.5 * rng.random(n - 1))
    return np.concatenate([[0.0], np.cumsum(h)]) - 0.5 * h.sum()


def make_case(name, dims, mode, freq, seed, dipoles):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    xn, yn, zn = graded(nx, 100.0, rng), graded(ny, 120.0, rng), graded(nz, 80.0, rng)
    cshape = (nx - 1, ny - 1, nz - 1)
    sig_re = (10.0 ** rng.uniform(-3, 0, cshape)).astype(np.float32)
    sig_re[:, :, :2] = 1e-8  # air on top
    eps_rel = rng.uniform(1, 30, cshape).astype(np.float32)
    eta = rng.uniform(0.05, 0.5, cshape).astype(np.float32)
    tau = (10.0 ** rng.uniform(-3, 0, cshape)).astype(np.float32)
    cee = rng.uniform(0.2, 0.8, cshape).astype(np.float32)
    omega = 2.0 * np.pi * freq
    sig = sigma_hat(mode, omega, sig_re, eps_rel, eta, tau, cee)
    k2 = np.concatenate([a.ravel(order="F") for a in wavenumbers(xn, yn, zn, sig, omega)])
    K = assemble(xn, yn, zn, k2)
    diag = jacobi_diag(xn, yn, zn, k2)
    n = K.shape[0]
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = K @ x
    b, nskip = rhs_mode5(xn, yn, zn, dipoles)
    # direct solve on the rows that are not identically zero (boundary Phi)
    B = Blocks(nx, ny, nz)
    live = np.asarray(abs(K).sum(axis=1)).ravel() > 0
    sol = np.zeros(n, complex)
    sol[live] = spla.spsolve(K[live][:, live].tocsc(), b[live])
    xq, iters, hist, conv = qmr_np(K, diag, b, 1e-10, 3000)
    bf, ef = fields(xn, yn, zn, omega, xq)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"), xn=xn, yn=yn, zn=zn, mode=mode, freq=freq,
        omega=omega, sig_re=sig_re.ravel(order="F"), eps_rel=eps_rel.ravel(order="F"),
        eta=eta.ravel(order="F"), tau=tau.ravel(order="F"), cee=cee.ravel(order="F"),
        sig=sig.ravel(order="F"), k2=k2, diag=diag, x=x, y=y, rhs=b, nskip=nskip,
        dip_dirs=np.array([d[0] for d in dipoles]), dip_ijk=np.array([d[1:] for d in dipoles]),
        sol_direct=sol, qmr_x=xq, qmr_iters=iters, qmr_hist=hist, qmr_conv=conv,
        fields_B=bf, fields_E=ef)
    print("%-10s dims=%s n=%d iters=%d conv=%s nskip=%d" % (name, dims, n, iters, conv, nskip))


CASES = [
    ("case_r", (6, 7, 8), "R", 1.0, 11,
     [("+X", 3, 4, 3), ("-Y", 2, 3, 4), ("+Z", 4, 4, 5), ("+Q", 1, 1, 1), ("+X", 6, 1, 1)]),
    ("case_c", (7, 6, 9), "C", 1.0e4, 12, [("+Y", 3, 3, 4), ("-X", 4, 2, 5), ("-Z", 2, 2, 1)]),
    ("case_d", (8, 8, 7), "D", 10.0, 13, [("+X", 4, 4, 3), ("-Z", 3, 5, 4)]),
    ("case_i", (5, 6, 6), "I", 1.0e6, 14, [("+Z", 3, 3, 2), ("-Y", 3, 5, 3)]),
]

if __name__ == "__main__":
    for c in CASES:
        make_case(*c)
    sys.exit(0)
