"""Host-side model setup: the reference's file formats, sigma-hat, sources,
and the seeded synthetic models the benchmarks run on.

File formats follow the reference's readers: aphid.input
(src/aphid.f90:183-252), aphid.mesh (:269-449), aphid.source (:638-741),
aphid_mpi.freq / aphid_mpi.input / aphid_mpi.source
(src/aphid_parallel.f90:45-104).  Arrays are Fortran-ordered and cell
properties are real(4), as read_mesh declares them (src/aphid.f90:288).
"""
import math
import re

import numpy as np

PI = 3.141592653589793
MU0 = PI * 4.0e-7            # src/aphid_mod.f90:10
EPS0 = 8.8541878176e-12      # src/aphid_mod.f90:12


# ------------------------------------------------------------------ mesh
def spacings(xn):
    """Node coordinates -> dx(0:n) (n+1 values) and dxc(1:n) (n values),
    src/aphid.f90:347-361."""
    xn = np.asarray(xn, dtype=np.float64)
    n = len(xn)
    if n < 3:
        raise ValueError("need at least 3 nodes per axis")
    d = np.empty(n + 1)
    d[1:n] = xn[1:] - xn[:-1]
    d[0], d[n] = d[1], d[n - 1]
    dc = np.empty(n)
    dc[1:n - 1] = 0.5 * (d[1:n - 1] + d[2:n])
    dc[0], dc[n - 1] = dc[1], dc[n - 2]
    return d, dc


def nunk(nx, ny, nz):
    return (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1) + nx * ny * nz


def block_offsets(nx, ny, nz):
    oy = (nx - 1) * ny * nz
    oz = oy + nx * (ny - 1) * nz
    op = oz + nx * ny * (nz - 1)
    return [0, oy, oz, op, op + nx * ny * nz]


def sigma_hat(mode, omega, sig_re=None, eps_rel=None, eta=None, tau=None, cee=None):
    """Complex cell conductivity for csig_flag R/C/D/I (src/aphid.f90:379-449).
    Inputs are rounded to real(4) as the reference reads them."""
    f = lambda a: None if a is None else np.asarray(a, dtype=np.float32).astype(np.float64)
    s, e, et, ta, c = f(sig_re), f(eps_rel), f(eta), f(tau), f(cee)
    w = 1j * omega
    if mode == "R":
        return s + w * EPS0
    if mode == "C":
        return s + w * EPS0 * e
    if mode == "D":
        return s * (1.0 - et / (1.0 + (w * ta) ** c))
    if mode == "I":
        return w * EPS0 * e
    raise ValueError("conductivity model must be R, C, D or I, got %r" % mode)


def gen_rhs(xn, yn, zn, mode, dipoles=()):
    """Right-hand side for oper_mode 1, 2, 3, 5 (src/aphid.f90:534-743) as a
    complex128 vector [Ax|Ay|Az|Phi].  Mode-5 dipoles are (dir, i, j, k) with
    the reference's 1-based tail-end node; out-of-range or invalid dipoles
    are skipped as the reference does.  Returns (b, n_skipped)."""
    xn, yn, zn = (np.asarray(a, float) for a in (xn, yn, zn))
    nx, ny, nz = len(xn), len(yn), len(zn)
    d = [spacings(xn)[0], spacings(yn)[0], spacings(zn)[0]]
    off = block_offsets(nx, ny, nz)
    shapes = [(nx - 1, ny, nz), (nx, ny - 1, nz), (nx, ny, nz - 1), (nx, ny, nz)]
    blk = [np.zeros(s, complex, order="F") for s in shapes]
    skipped = 0
    if mode == 1:
        tol = float(np.float32(1e-4))
        hit = lambda c: [i for i in range(len(c)) if abs(c[i]) < tol]
        ix, jy, kz = hit(xn), hit(yn), hit(zn)
        if not (ix and jy and kz) or ix[-1] > nx - 2:
            raise ValueError("mode 1 needs a mesh node at the origin")
        i, j, k = ix[-1], jy[-1], kz[-1]
        blk[0][i, j, k] = MU0
        blk[3][i, j, k] = MU0 / d[0][i + 1]
        blk[3][i + 1, j, k] = -MU0 / d[0][i + 1]
    elif mode == 2:
        blk[0][:, :, 1] = MU0 * d[0][1:nx][:, None] * (0.5 * (d[1][0:ny] + d[1][1:ny + 1]))[None, :]
    elif mode == 3:
        blk[1][:, :, 1] = MU0 * d[1][1:ny][None, :] * (0.5 * (d[0][0:nx] + d[0][1:nx + 1]))[:, None]
    elif mode == 5:
        lim = [nx, ny, nz]
        for dr, i, j, k in dipoles:
            dr = str(dr)
            if len(dr) != 2 or dr[0] not in "+-" or dr[1] not in "XYZ":
                skipped += 1
                continue
            a = "XYZ".index(dr[1])
            tail = [int(i) - 1, int(j) - 1, int(k) - 1]
            if dr[0] == "-":
                tail[a] -= 1  # "-X i j k" is the edge (i-1, i) with reversed sign
            head = list(tail)
            head[a] += 1
            ok = all(0 <= t < (lim[q] - 1 if q == a else lim[q]) for q, t in enumerate(tail))
            if not ok:
                skipped += 1
                continue
            sgn = 1.0 if dr[0] == "+" else -1.0
            blk[a][tuple(tail)] += sgn * MU0 * d[a][tail[a] + 1]
            blk[3][tuple(tail)] += sgn * MU0
            blk[3][tuple(head)] -= sgn * MU0
    else:
        raise ValueError("oper_mode %r not supported here" % mode)
    b = np.concatenate([x.ravel(order="F") for x in blk])
    return b, skipped


# ----------------------------------------------------------- file formats
_num = re.compile(r"[-+]?(\d+\.?\d*|\.\d+)([eEdD][-+]?\d+)?")


def _fnum(tok):
    return float(tok.replace("d", "e").replace("D", "e"))


def _first(line):
    return line.split("!")[0].split()[0]


def read_input(path):
    """aphid.input: 3 header lines, then oper_mode, qmr_target, qmr_max_it,
    freq, csig_flag (src/aphid.f90:194-216)."""
    with open(path) as f:
        lines = f.read().splitlines()
    if len(lines) < 8:
        raise ValueError("aphid.input: expected 8 lines")
    out = dict(oper_mode=int(_first(lines[3])), qmr_target=_fnum(_first(lines[4])),
               qmr_max_it=int(_first(lines[5])), freq=_fnum(_first(lines[6])),
               csig_flag=_first(lines[7])[0].upper())
    if out["qmr_target"] < 0:
        raise ValueError("Invalid target residual: value must positive.")
    if out["qmr_max_it"] < 0:
        raise ValueError("Invalid qmr_max_it: value must positive.")
    out["omega"] = 2.0 * PI * out["freq"]
    return out


def write_input(path, oper_mode, qmr_target, qmr_max_it, freq, csig_flag="R"):
    bar = "=" * 72
    with open(path, "w") as f:
        f.write("%s\nAPHID Input File: operational parameters\n%s\n" % (bar, bar))
        f.write("%-10d!! operational mode\n" % oper_mode)
        f.write("%-10.3e!! QMR target residual\n" % qmr_target)
        f.write("%-10d!! max QMR iterates\n" % qmr_max_it)
        f.write("%-10.6e!! frequency [Hz]\n" % freq)
        f.write("%-10s!! conductivity model: [R]eal, [C]omplex, [D]ispersive, [I]nsulator\n"
                % csig_flag)


class _Records:
    """Fortran list-directed reading: each READ starts on a new record and
    consumes as many records as it needs values."""

    def __init__(self, text):
        self.lines = text.splitlines()
        self.pos = 0

    def skip(self):
        self.pos += 1

    def read(self, count, conv=float):
        vals = []
        while len(vals) < count:
            if self.pos >= len(self.lines):
                raise ValueError("unexpected end of file")
            toks = self.lines[self.pos].replace(",", " ").split()
            self.pos += 1
            vals.extend(toks)
        return np.array([conv(_fnum(t)) if conv is float else conv(t) for t in vals[:count]])


def read_mesh(path, csig_flag="R"):
    """aphid.mesh (src/aphid.f90:316-449).  Returns a dict with node
    coordinates and the real(4) cell arrays the conductivity model needs."""
    with open(path) as f:
        r = _Records(f.read())
    nx, ny, nz = (int(v) for v in r.read(3, conv=int))
    r.skip()
    xn = r.read(nx)
    r.skip()
    yn = r.read(ny)
    r.skip()
    zn = r.read(nz)
    nc = (nx - 1) * (ny - 1) * (nz - 1)
    names = {"R": ["sig_re"], "C": ["sig_re", "eps_rel"], "D": ["sig_re", "eta", "tau", "cee"],
             "I": ["eps_rel"]}[csig_flag]
    out = dict(xn=xn, yn=yn, zn=zn)
    for name in names:
        r.skip()
        out[name] = r.read(nc).astype(np.float32)
    return out


def write_mesh(path, xn, yn, zn, sig_re=None, eps_rel=None, eta=None, tau=None, cee=None):
    """Writes aphid.mesh in the layout of serial/gen_mesh.f90 (6 values per
    line, section header lines) so read_mesh and the reference read it."""
    def block(f, a):
        a = np.asarray(a).ravel(order="F")
        for s in range(0, len(a), 6):
            f.write(" ".join("%13.6e" % v for v in a[s:s + 6]) + "\n")
    with open(path, "w") as f:
        f.write(" %d %d %d\n \n" % (len(xn), len(yn), len(zn)))
        block(f, xn)
        f.write(" \n")
        block(f, yn)
        f.write(" \n")
        block(f, zn)
        for title, arr in (("REAL CONDUCTIVITY", sig_re), ("RELATIVE ELECTRIC PERMITTIVITY", eps_rel),
                           ("CHARGEABILITY", eta), ("TIME CONSTANT", tau),
                           ("FREQUENCY EXPONENT", cee)):
            if arr is not None:
                f.write(" %s\n" % title)
                block(f, np.asarray(arr, dtype=np.float32))


def read_source(path):
    """aphid.source: one dipole per line, `dir i j k` (src/aphid.f90:640-646)."""
    out = []
    with open(path) as f:
        for line in f:
            t = line.split("!")[0].split()
            if len(t) >= 4:
                out.append((t[0], int(t[1]), int(t[2]), int(t[3])))
    return out


def write_source(path, dipoles):
    with open(path, "w") as f:
        for d, i, j, k in dipoles:
            f.write("%s %d %d %d\n" % (d, i, j, k))


def read_mpi_freq(path):
    """aphid_mpi.freq: 3 header lines, a count, then one frequency per line
    (src/aphid_parallel.f90:45-53)."""
    with open(path) as f:
        lines = f.read().splitlines()
    n = int(_first(lines[3]))
    return np.array([_fnum(_first(lines[4 + q])) for q in range(n)])


def read_mpi_input(path):
    """aphid_mpi.input: 'MT' or 'CS', target, max iterations, model flag."""
    with open(path) as f:
        lines = f.read().splitlines()
    return dict(source_type=_first(lines[3])[:2].upper(), qmr_target=_fnum(_first(lines[4])),
                qmr_max_it=int(_first(lines[5])), csig_flag=_first(lines[6])[0].upper())


def read_mpi_source(path):
    """aphid_mpi.source: list of dipole arrays (src/aphid_parallel.f90:90-95,
    168-193): a count, then per array a header block, its dipole count and
    its dipoles."""
    with open(path) as f:
        lines = [l.split("!")[0].strip() for l in f.read().splitlines()]
    data = [l for l in lines[3:] if l and not l.startswith("=") and not l.lower().startswith("dipole")
            and not l.lower().startswith("aphid")]
    n = int(data[0].split()[0])
    pos, arrays = 1, []
    for _ in range(n):
        m = int(data[pos].split()[0])
        pos += 1
        arr = []
        for _ in range(m):
            t = data[pos].split()
            arr.append((t[0], int(t[1]), int(t[2]), int(t[3])))
            pos += 1
        arrays.append(arr)
    return arrays


def write_mpi_freq(path, freqs):
    """aphid_mpi.freq in the layout read_mpi_freq (and the farm) reads"""
    bar = "=" * 72
    with open(path, "w") as f:
        f.write("%s\nAPHID: source frequency array [Hz]\n%s\n" % (bar, bar))
        f.write("%-13d! number of frequencies\n" % len(freqs))
        for v in freqs:
            f.write("%-13.6e\n" % v)


def write_mpi_input(path, source_type, qmr_target, qmr_max_it, csig_flag="R"):
    """aphid_mpi.input: MT or CS, QMR target, iteration cap, model flag"""
    bar = "=" * 72
    with open(path, "w") as f:
        f.write("%s\nAPHID Input File: Operational parameters for PARALLEL MPI computation\n%s\n" % (bar, bar))
        f.write("%-10s!! mode of operation (either 'MT', or 'CS' for dipole array)\n" % source_type)
        f.write("%-10.3e!! QMR target residual\n" % qmr_target)
        f.write("%-10d!! max QMR iterates\n" % qmr_max_it)
        f.write("%-10s!! conductivity model: [R]eal, [C]omplex, [D]ispersive, [I]nsulator\n" % csig_flag)


def write_mpi_source(path, arrays):
    """aphid_mpi.source: the dipole arrays of a CS sweep, each a list of
    (dir, i, j, k), in the block layout the farm reads"""
    bar = "=" * 72
    with open(path, "w") as f:
        f.write("%s\nAPHID: list of controlled-source electric dipole array sources\n%s\n" % (bar, bar))
        f.write("%-15d!  number of dipole arrays\n\n" % len(arrays))
        for arr in arrays:
            f.write("%s\ndipole array definition\n%s\n" % (bar, bar))
            f.write("%-15d! number of elementary dipoles in array\n" % len(arr))
            for d, i, j, k in arr:
                f.write("%s %d %d %d\n" % (d, i, j, k))
            f.write("\n")


def sweep_systems(freqs, source_type, dipole_arrays=None):
    """The (frequency, source) list the MPI farm distributes
    (src/aphid_parallel.f90:75-103): MT gives modes 2 and 3 per frequency,
    CS gives mode 5 per dipole array; frequencies vary fastest."""
    systems = []
    if source_type == "MT":
        for mode in (2, 3):
            systems += [dict(freq=f, mode=mode, dipoles=()) for f in freqs]
    else:
        for arr in dipole_arrays:
            systems += [dict(freq=f, mode=5, dipoles=tuple(arr)) for f in freqs]
    return systems


# --------------------------------------------------------- synthetic models
def graded_axis(ncell, core=1000.0, npad=6, ratio=1.3):
    """Cell widths: `ncell - 2*npad` uniform core cells, `npad` cells on each
    side growing geometrically by `ratio`; nodes centred on 0."""
    ncore = ncell - 2 * npad
    if ncore < 1:
        raise ValueError("too few cells for the padding")
    pad = core * ratio ** np.arange(1, npad + 1)
    h = np.concatenate([pad[::-1], np.full(ncore, core), pad])
    x = np.concatenate([[0.0], np.cumsum(h)])
    return x - 0.5 * x[-1]


def depth_axis(ncell, nair, core=1000.0, npad=6, ratio=1.3):
    """Same grading along z (positive down), z = 0 at node `nair`
    (0-based), the top of the first earth cell."""
    z = graded_axis(ncell, core, npad, ratio)
    return z - z[nair]


def grf(shape, corr, rng):
    """Zero-mean, unit-variance Gaussian random field with Gaussian
    covariance exp(-r^2/corr^2) (cells), by FFT filtering of white noise."""
    w = rng.standard_normal(shape)
    k = np.meshgrid(*[2 * np.pi * np.fft.fftfreq(n) for n in shape], indexing="ij")
    k2 = sum(kk ** 2 for kk in k)
    f = np.fft.ifftn(np.fft.fftn(w) * np.exp(-k2 * corr ** 2 / 8.0)).real
    f -= f.mean()
    return f / f.std()


class Model:
    """A synthetic problem: mesh, real(4) cell conductivity, sources and
    frequencies."""

    def __init__(self, name, xn, yn, zn, sig_re, freqs, sources, target=1e-8, csig_flag="R",
                 eps_rel=None):
        self.name, self.xn, self.yn, self.zn = name, xn, yn, zn
        self.sig_re = np.asarray(sig_re, np.float32)
        self.eps_rel = eps_rel
        self.freqs = np.atleast_1d(np.asarray(freqs, float))
        self.sources = sources      # list of dipole lists (mode 5)
        self.target = target
        self.csig_flag = csig_flag

    @property
    def dims(self):
        return len(self.xn), len(self.yn), len(self.zn)

    @property
    def n(self):
        return nunk(*self.dims)

    @property
    def ncell(self):
        nx, ny, nz = self.dims
        return (nx - 1) * (ny - 1) * (nz - 1)

    def systems(self):
        return [(f, s) for s in range(len(self.sources)) for f in self.freqs]


def _earth(cshape, nair, rng, nblocks=20, corr=8.0):
    sig = np.full(cshape, 1e-8)
    ez = cshape[2] - nair
    u = np.clip(-2.0 + grf((cshape[0], cshape[1], ez), corr, rng), -4.0, 1.0)
    e = 10.0 ** u
    for _ in range(nblocks):
        lo = [int(rng.integers(0, max(1, c - 4))) for c in (cshape[0], cshape[1], ez)]
        sz = [int(rng.integers(2, 13)) for _ in range(3)]
        e[lo[0]:lo[0] + sz[0], lo[1]:lo[1] + sz[1], lo[2]:lo[2] + sz[2]] = 10.0 ** rng.uniform(-4, 1)
    sig[:, :, nair:] = e
    return sig


def _e12_4(v):
    """values as Fortran's e12.4 edit descriptor prints them (5 significant
    digits), which is how gen_mesh.f90 writes aphid.mesh"""
    return np.array([float("%12.4e" % x) for x in np.asarray(v, np.float32)])


def serial_mt_model(nh=50):
    """The reference's serial MT example (serial/gen_mesh.f90), the 1-D
    layered-earth check of the paper: nh x nh x 121 nodes.  Horizontally
    uniform 200 km / 49 cells (nh = 50 reproduces the file; any nh >= 3
    gives the same laterally uniform solution under an MT sheet source).
    Vertically 51 air cells of 100 km / 51 above z = 0, then 19 cells of
    1 km, 20 of 50 m and 30 of 1 km down to 50 km, node coordinates
    accumulated in real(4) and rounded as e12.4 writes them.  Cell
    conductivity by cell-centre depth: air 1e-8 S/m, 0.001 S/m down to
    19 km, 0.1 S/m to 20 km, 0.01 S/m below (gen_mesh.f90's loop, in which
    the shallower conditions override the deeper ones).  Returns (xn, yn,
    zn, sig_re (nh-1, nh-1, 120) real(4), index of the surface node)."""
    nair, near = 51, 69
    z = np.zeros(nair + near + 1, np.float32)
    z[0] = -100e3
    dza = np.float32(100e3) / np.float32(nair)
    for i in range(1, nair + 1):
        z[i] = z[i - 1] + dza
    for i in range(nair + 1, nair + near + 1):
        f = i + 1  # Fortran index
        small = nair + 2 + 19 <= f < nair + 41
        z[i] = z[i - 1] + (np.float32(50.0) if small else np.float32(1e3))
    h = np.float32(200e3) / np.float32(49)
    x = np.float32(-100e3) + h * np.arange(nh, dtype=np.float32)
    zc = 0.5 * (z[:-1] + z[1:])
    sc = np.full(zc.shape, 0.01, np.float32)
    sc[zc < 20e3] = 0.10
    sc[zc < 19e3] = 0.001
    sc[zc < 0.0] = 1e-8
    sig = np.broadcast_to(sc[None, None, :], (nh - 1, nh - 1, len(zc))).astype(np.float32)
    return _e12_4(x), _e12_4(x), _e12_4(z), np.asfortranarray(sig), nair


def make_model(config, seed=None):
    """Seeded synthetic stand-ins for the benchmark configurations.

    halfspace32   32^3 cells, 8 air layers over a 0.01 S/m half-space, one +X
                  dipole at the centre of the surface, 1 Hz
    hetero96      96^3 cells, Gaussian-random-field earth (corr. 8 cells,
                  mean -2, std 1, clipped to [-4, 1] in log10) + 20 blocks,
                  8 air layers, +X dipole at the surface, 1 Hz
    sweep128      128x128x96 cells, heterogeneous earth, 24 frequencies
                  log-spaced 1e-3..1e5 Hz x 4 surface dipoles (96 systems)
    train64 / eval160   64x64x48 / 160x160x128 heterogeneous (learned guess)
    seafloor256   256x256x192 cells, 10 air layers, 15 seawater layers at
                  3.3 S/m, heterogeneous earth, 24 frequencies, one +X dipole
                  on the seafloor
    seafloor96    the same layering on 96^3 cells at 0.272 Hz, where the
                  complex64 Lanczos form collapses (escalation test case)
    """
    cfg = {
        "halfspace32": (32, 32, 32, 8, 0, 1),
        "hetero96": (96, 96, 96, 8, 0, 2),
        "sweep128": (128, 128, 96, 8, 0, 3),
        "train64": (64, 64, 48, 8, 0, 4),
        "eval160": (160, 160, 128, 8, 0, 5),
        "seafloor256": (256, 256, 192, 10, 15, 6),
        "seafloor96": (96, 96, 96, 10, 15, 6),
    }
    if config not in cfg:
        raise KeyError("unknown synthetic model %r" % config)
    cx, cy, cz, nair, nsea, default_seed = cfg[config]
    rng = np.random.default_rng(default_seed if seed is None else seed)
    xn, yn = graded_axis(cx), graded_axis(cy)
    zn = depth_axis(cz, nair)
    cshape = (cx, cy, cz)
    if config == "halfspace32":
        sig = np.full(cshape, 0.01)
        sig[:, :, :nair] = 1e-8
    else:
        sig = _earth(cshape, nair + nsea, rng)
        sig[:, :, nair:nair + nsea] = 3.3
    ic, jc = cx // 2, (cy + 2) // 2          # 1-based: edge (ic, ic+1) straddles x = 0
    ks = nair + nsea + 1                      # 1-based node on the earth's (or sea floor's) top
    if config == "sweep128":
        off = cx // 8
        sources = [[("+X", ic, jc, ks)], [("+Y", ic + 1, jc - 1, ks)],
                   [("+X", ic + off, jc + off, ks)], [("+Y", ic + off + 1, jc + off - 1, ks)]]
        freqs = np.logspace(-3, 5, 24)
    elif config == "seafloor256":
        sources = [[("+X", ic, jc, ks)]]
        freqs = np.logspace(-3, 5, 24)
    elif config == "seafloor96":
        sources = [[("+X", ic, jc, ks)]]
        freqs = [0.272]
    else:
        sources = [[("+X", ic, jc, ks)]]
        freqs = [1.0]
    return Model(config, xn, yn, zn, sig.astype(np.float32), freqs, sources)
