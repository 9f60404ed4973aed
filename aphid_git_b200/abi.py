"""ctypes binding of the C ABI (include/aphid_gpu.h).

The names mirror the reference's routines (src/aphid.f90, src/aphid_qmr.f90):
``inprod`` (inprod_x/y/z/p), ``gen_k2`` (gen_k2_*grid), ``gen_diag``,
``qmr`` and ``gen_fields``.  Vectors are numpy complex128 arrays in the
reference's unknown order [Ax | Ay | Az | Phi], each block Fortran-ordered.

There is no CPU fallback: if libaphid_gpu.so is missing or no sm_100 device
is present, every entry point raises.
"""
import ctypes as C
import os

import numpy as np

from . import build as _build

APHID_OK = 0
STATUS = {0: "converged", 1: "maxit", 2: "breakdown", 3: "nonfinite"}
ERRORS = {-1: "bad argument", -2: "CUDA error", -3: "out of device memory",
          -4: "call order", -5: "no sm_100 device"}
PREC_FP64, PREC_MIXED, PREC_FUSED64, PREC_AUTO = 0, 1, 2, 3
PRECISIONS = {"fp64": PREC_FP64, "mixed": PREC_MIXED, "fused64": PREC_FUSED64, "auto": PREC_AUTO}


class AphidError(RuntimeError):
    pass


class SweepOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("target", C.c_double), ("max_it", C.c_int),
                ("inner_tol", C.c_double), ("max_outer", C.c_int), ("stall_window", C.c_int),
                ("reserved", C.c_int * 2)]


class Source(C.Structure):
    """aphid_source: oper_mode 2 / 3 (MT sheet sources) or 5 (dipole list)"""
    _fields_ = [("oper_mode", C.c_int), ("ndip", C.c_int), ("dip_dir", C.c_char_p),
                ("dip_ijk", C.c_void_p)]


class GroupJob(C.Structure):
    """aphid_group_job: one context's part of a group sweep"""
    _fields_ = [("ctx", C.c_void_p), ("nsys", C.c_int), ("omega", C.c_void_p),
                ("source_of_system", C.c_void_p), ("nsrc", C.c_int), ("srcs", C.c_void_p),
                ("x0", C.c_void_p), ("x_out", C.c_void_p), ("info", C.c_void_p)]


class Opts(C.Structure):
    _fields_ = [("device", C.c_int), ("stream", C.c_void_p), ("graph_iters", C.c_int),
                ("verbose", C.c_int), ("plane_kz", C.c_int)]


class Info(C.Structure):
    _fields_ = [("status", C.c_int), ("iters", C.c_int), ("inner_iters", C.c_int),
                ("outer_iters", C.c_int), ("rhs_norm", C.c_double), ("recur_resid", C.c_double),
                ("true_rel_resid", C.c_double), ("seconds", C.c_double),
                ("kernel_launches", C.c_longlong), ("inner64_iters", C.c_int)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["status_name"] = STATUS.get(self.status, str(self.status))
        return d


_lib = None
_Z = C.c_void_p


def library_path():
    return _build.LIB


def load():
    """Load libaphid_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise AphidError("libaphid_gpu.so not built: run `python -m aphid_git_b200.build`")
    L = C.CDLL(path)
    P = C.c_void_p
    L.aphid_gpu_create.argtypes = [C.POINTER(P), C.POINTER(Opts)]
    L.aphid_gpu_destroy.argtypes = [P]
    L.aphid_gpu_last_error.argtypes = [P]
    L.aphid_gpu_last_error.restype = C.c_char_p
    L.aphid_gpu_set_mesh.argtypes = [P, C.c_int, C.c_int, C.c_int] + [P] * 6
    L.aphid_gpu_inprod.argtypes = [P] + [_Z] * 12
    L.aphid_gpu_gen_k2.argtypes = [P, _Z, C.c_double] + [_Z] * 4
    L.aphid_gpu_gen_diag.argtypes = [P] + [_Z] * 8
    L.aphid_gpu_qmr.argtypes = [P] + [_Z] * 16 + [C.c_double, C.c_int, P, C.c_int,
                                                   C.POINTER(Info)]
    L.aphid_gpu_fields.argtypes = [P, C.c_double] + [_Z] * 10
    L.aphid_gpu_qmr_load.argtypes = [P] + [_Z] * 12
    L.aphid_gpu_qmr_run.argtypes = [P, C.c_double, C.c_int, C.c_int, P, C.c_int, C.POINTER(Info)]
    L.aphid_gpu_qmr_fetch.argtypes = [P] + [_Z] * 4
    L.aphid_gpu_inprod_dev.argtypes = [P, P, P, P, P]
    L.aphid_gpu_inprod_eps_noalloc.argtypes = [C.c_int] * 3 + [P] * 11
    L.aphid_gpu_set_model.argtypes = [P, C.c_char, P, P]
    L.aphid_gpu_set_model_cole_cole.argtypes = [P, P, P, P, P]
    L.aphid_gpu_sweep.argtypes = [P, C.c_int, P, P, C.c_int, P, C.c_char_p, P, P,
                                  C.POINTER(SweepOpts), P, P]
    L.aphid_gpu_sweep_sources.argtypes = [P, C.c_int, P, P, C.c_int, P, P, C.POINTER(SweepOpts), P, P]
    L.aphid_gpu_sweep_receivers.argtypes = [P, C.c_int, P, P, P]
    L.aphid_gpu_sweep_group.argtypes = [C.c_int, P, C.POINTER(SweepOpts)]
    L.aphid_gpu_sweep_fetch.argtypes = [P, C.c_int, P]
    L.aphid_gpu_sweep_time_apply.argtypes = [P, C.c_int]
    L.aphid_gpu_sweep_apply.argtypes = [P, _Z, _Z]
    L.aphid_gpu_sweep_plane_kz.argtypes = [P]
    L.aphid_gpu_sweep_pass_config.argtypes = [P]
    L.aphid_gpu_sweep_tile_shape.argtypes = [P]
    _lib = L
    return L


def nunk(nx, ny, nz):
    return (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1) + nx * ny * nz


def block_offsets(nx, ny, nz):
    ox = 0
    oy = (nx - 1) * ny * nz
    oz = oy + nx * (ny - 1) * nz
    op = oz + nx * ny * (nz - 1)
    return [ox, oy, oz, op, op + nx * ny * nz]


def _c128(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if n is not None and a.size != n:
        raise ValueError("expected %d complex values, got %d" % (n, a.size))
    return a


def _sources(sources):
    """aphid_source array for a list of sources (dipole lists or the MT
    oper_mode 2 / 3); returns (array, buffers to keep alive)"""
    arr = (Source * len(sources))()
    keep = []
    for q, src in enumerate(sources):
        if isinstance(src, (int, np.integer)) and not isinstance(src, bool):
            if int(src) not in (2, 3):
                raise AphidError("an integer source must be oper_mode 2 or 3 (MT), got %r" % (src,))
            arr[q].oper_mode = int(src)
            continue
        dips = list(src)
        dirs = "".join(str(d[0])[:2].ljust(2) for d in dips).encode() or b"  "
        ijk = np.array([[int(d[1]), int(d[2]), int(d[3])] for d in dips] or [[0, 0, 0]], dtype=np.int32)
        keep += [dirs, ijk]
        arr[q].oper_mode = 5
        arr[q].ndip = len(dips)
        arr[q].dip_dir = dirs
        arr[q].dip_ijk = ijk.ctypes.data
    return arr, keep


NOALLOC_MAX_NODES = 1024
NOALLOC_MAX_SLOTS = 16384


def inprod_eps_noalloc(nx, ny, nz, d_spacing, d_k2, d_in, d_out, d_eps, stream=0):
    """Allocation-free y = K x with epsilon = x^T y (aphid_gpu_inprod_eps_noalloc).

    For callers that cannot allocate device memory: every argument is a device
    pointer the caller owns (d_spacing = six pointers dx, dy, dz, dxc, dyc,
    dzc), and the scratch is a fixed array inside the library, shared by all
    calls (overlapping calls race).  Meshes above NOALLOC_MAX_NODES nodes per
    axis are rejected.  Asynchronous on `stream`; returns the status code."""
    return load().aphid_gpu_inprod_eps_noalloc(nx, ny, nz, *d_spacing, d_k2, d_in, d_out, d_eps,
                                               stream)


class Solver:
    """One GPU context (one per host thread), bound to a mesh."""

    def __init__(self, device=0, stream=None, graph_iters=0, verbose=False, plane_kz=0):
        self.lib = load()
        self._h = C.c_void_p()
        o = Opts(device, stream or 0, graph_iters, int(verbose), plane_kz)
        rc = self.lib.aphid_gpu_create(C.byref(self._h), C.byref(o))
        if rc != APHID_OK:
            raise AphidError("aphid_gpu_create failed: %s" % ERRORS.get(rc, rc))
        self.dims = None
        self._last_nsys = 0

    def close(self):
        if self._h:
            self.lib.aphid_gpu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc != APHID_OK:
            msg = self.lib.aphid_gpu_last_error(self._h).decode()
            raise AphidError("%s: %s (%s)" % (what, ERRORS.get(rc, rc), msg))

    # ------------------------------------------------------------- mesh
    def set_mesh(self, dx, dy, dz, dxc, dyc, dzc):
        """dx(0:n), dxc(1:n) per axis (the reference's module mesh arrays)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (dx, dy, dz, dxc, dyc, dzc)]
        nx, ny, nz = len(arrs[3]), len(arrs[4]), len(arrs[5])
        if [len(a) for a in arrs[:3]] != [nx + 1, ny + 1, nz + 1]:
            raise ValueError("dx must have n+1 values and dxc n values per axis")
        self._keep = arrs
        self._check(self.lib.aphid_gpu_set_mesh(self._h, nx, ny, nz,
                                                *[a.ctypes.data for a in arrs]), "set_mesh")
        self.dims = (nx, ny, nz)
        self.n = nunk(nx, ny, nz)
        self.off = block_offsets(nx, ny, nz)

    def set_nodes(self, xn, yn, zn):
        from .model import spacings
        (dx, dxc), (dy, dyc), (dz, dzc) = spacings(xn), spacings(yn), spacings(zn)
        self.set_mesh(dx, dy, dz, dxc, dyc, dzc)
        self.xn, self.yn, self.zn = (np.asarray(v, np.float64) for v in (xn, yn, zn))

    def _blocks(self, v):
        b = v.ctypes.data
        return [b + 16 * o for o in self.off[:4]]

    # --------------------------------------------------------- operators
    def inprod(self, k2, x):
        """y = K x (inprod_x, inprod_y, inprod_z, inprod_p)."""
        k2, x = _c128(k2, self.n), _c128(x, self.n)
        y = np.empty(self.n, np.complex128)
        self._check(self.lib.aphid_gpu_inprod(self._h, *self._blocks(k2), *self._blocks(x),
                                              *self._blocks(y)), "inprod")
        return y

    def gen_k2(self, sig, omega):
        nx, ny, nz = self.dims
        sig = _c128(sig, (nx - 1) * (ny - 1) * (nz - 1))
        k2 = np.empty(self.n, np.complex128)
        self._check(self.lib.aphid_gpu_gen_k2(self._h, sig.ctypes.data, float(omega),
                                              *self._blocks(k2)), "gen_k2")
        return k2

    def gen_diag(self, k2):
        k2 = _c128(k2, self.n)
        d = np.empty(self.n, np.complex128)
        self._check(self.lib.aphid_gpu_gen_diag(self._h, *self._blocks(k2), *self._blocks(d)),
                    "gen_diag")
        return d

    def qmr(self, k2, diag, b, target, max_it, x0=None, hist=True):
        """Solve K x = b like `call qmr`.  Returns (x, info dict, hist array)."""
        k2, diag = _c128(k2, self.n), _c128(diag, self.n)
        x = _c128(b, self.n).copy()
        x0a = _c128(x0, self.n) if x0 is not None else None  # keep alive across the call
        x0p = self._blocks(x0a) if x0a is not None else [None] * 4
        cap = max(1, max_it) if hist else 0
        h = np.zeros(max(cap, 1))
        info = Info()
        self._check(self.lib.aphid_gpu_qmr(self._h, *self._blocks(k2), *self._blocks(diag),
                                           *self._blocks(x), *x0p, float(target), int(max_it),
                                           h.ctypes.data if hist else None, cap,
                                           C.byref(info)), "qmr")
        d = info.as_dict()
        nh = min(d["inner_iters"], cap)
        return x, d, h[:nh]

    def qmr_load(self, k2, diag, b):
        """Make k2, diag and b resident on the device (aphid_gpu_qmr_load)."""
        self._res = [_c128(k2, self.n), _c128(diag, self.n), _c128(b, self.n)]
        self._check(self.lib.aphid_gpu_qmr_load(self._h, *self._blocks(self._res[0]),
                                                *self._blocks(self._res[1]),
                                                *self._blocks(self._res[2])), "qmr_load")

    def qmr_run(self, target, max_it, use_previous_x=False, hist=False):
        """Solve the resident problem; the solution stays on the device."""
        cap = max(1, max_it) if hist else 0
        h = np.zeros(max(cap, 1))
        info = Info()
        self._check(self.lib.aphid_gpu_qmr_run(self._h, float(target), int(max_it),
                                               int(bool(use_previous_x)),
                                               h.ctypes.data if hist else None, cap,
                                               C.byref(info)), "qmr_run")
        d = info.as_dict()
        return d, h[:min(d["inner_iters"], cap)]

    def qmr_fetch(self):
        x = np.empty(self.n, np.complex128)
        self._check(self.lib.aphid_gpu_qmr_fetch(self._h, *self._blocks(x)), "qmr_fetch")
        return x

    def inprod_dev(self, d_k2, d_in, d_out, d_eps=None):
        """y = K x on device pointers (concatenated complex128 vectors);
        asynchronous on the context's stream."""
        self._check(self.lib.aphid_gpu_inprod_dev(self._h, d_k2, d_in, d_out, d_eps),
                    "inprod_dev")

    # ------------------------------------------------------------ sweep
    def set_model(self, csig_flag, sig_re=None, eps_rel=None):
        """Cell model for sweeps: 'R' (sig_re), 'C' (sig_re, eps_rel) or 'I'
        (eps_rel); real(4) cell arrays of (nx-1)(ny-1)(nz-1) values, Fortran
        order."""
        nx, ny, nz = self.dims
        nc = (nx - 1) * (ny - 1) * (nz - 1)

        def f32(a):
            if a is None:
                return None
            a = np.asarray(a, dtype=np.float32)
            a = np.ascontiguousarray(a.ravel(order="F") if a.ndim == 3 else a)
            if a.size != nc:
                raise ValueError("cell array must have %d values" % nc)
            return a
        self._model = [f32(sig_re), f32(eps_rel)]
        self._check(self.lib.aphid_gpu_set_model(
            self._h, csig_flag.encode(),
            self._model[0].ctypes.data if self._model[0] is not None else None,
            self._model[1].ctypes.data if self._model[1] is not None else None), "set_model")

    def set_model_cole_cole(self, sig_re, eta, tau, cee):
        """Cole-Cole cell model (csig_flag 'D'): real(4) cell arrays sigma,
        eta, tau, c; each sweep forms the averaged sigma-hat of every
        frequency on the device."""
        nx, ny, nz = self.dims
        nc = (nx - 1) * (ny - 1) * (nz - 1)
        arrs = []
        for a in (sig_re, eta, tau, cee):
            a = np.asarray(a, dtype=np.float32)
            a = np.ascontiguousarray(a.ravel(order="F") if a.ndim == 3 else a)
            if a.size != nc:
                raise ValueError("cell array must have %d values" % nc)
            arrs.append(a)
        self._model = arrs
        self._check(self.lib.aphid_gpu_set_model_cole_cole(self._h, *[a.ctypes.data for a in arrs]),
                    "set_model_cole_cole")

    def sweep(self, omegas, sources, source_of_system=None, x0=None, precision="auto",
              target=1e-8, max_it=20000, inner_tol=0.0, max_outer=0, stall_window=0, fetch=True,
              out=None):
        """Solve all (omega, source) systems in one batched launch.

        sources: one entry per source, each an oper_mode-5 dipole list
        [(dir, i, j, k), ...] or the integer 2 or 3 (the x- or y-polarised
        MT sheet source of gen_rhs); source_of_system[s] picks the source of
        system s (default: s).
        precision: "auto" (complex64 inner solves; systems whose Lanczos
        bilinear form collapses below complex64 resolution finish in
        complex128), "mixed", "fused64" (complex128 inner solves, same
        batched pass) or "fp64" (the reference's recurrence, one system at a
        time).
        out: an optional C-contiguous complex128 (nsys, nunk) array (pinned
        host memory makes the copy fastest) that receives the solutions.
        Returns (X, infos): X is (nsys, nunk) complex128 (None when fetch is
        False: the solutions stay on the device, see sweep_fetch)."""
        om = np.ascontiguousarray(np.atleast_1d(omegas), dtype=np.float64)
        nsys = om.size
        sos = np.ascontiguousarray(np.arange(nsys) if source_of_system is None
                                   else source_of_system, dtype=np.int32)
        srcs, keep = _sources(sources)
        x0a = None if x0 is None else np.ascontiguousarray(x0, dtype=np.complex128).reshape(nsys, self.n)
        if out is not None:
            if (out.dtype != np.complex128 or out.shape != (nsys, self.n) or not out.flags["C_CONTIGUOUS"]):
                raise AphidError("out must be a C-contiguous complex128 array of shape (%d, %d)" % (nsys, self.n))
            X = out
        else:
            X = np.empty((nsys, self.n), np.complex128) if fetch else None
        infos = (Info * nsys)()
        self._last_nsys = 0
        if precision not in PRECISIONS:
            raise AphidError("precision must be one of %s" % ", ".join(PRECISIONS))
        o = SweepOpts(PRECISIONS[precision], float(target), int(max_it),
                      float(inner_tol), int(max_outer), int(stall_window))
        self._check(self.lib.aphid_gpu_sweep_sources(
            self._h, nsys, om.ctypes.data, sos.ctypes.data, len(sources), srcs,
            x0a.ctypes.data if x0a is not None else None,
            C.byref(o), X.ctypes.data if X is not None else None, infos), "sweep")
        del keep
        self._last_nsys = nsys
        return X, [i.as_dict() for i in infos]

    def sweep_receivers(self, rec_ijk, e=True, h=True):
        """E and H at receiver nodes for every system of the last sweep
        (aphid_gpu_sweep_receivers): rec_ijk is (nrec, 3) 1-based interior
        nodes; returns (E, H), each (nsys, nrec, 3) complex128 or None."""
        rec = np.ascontiguousarray(np.atleast_2d(rec_ijk), dtype=np.int32)
        if rec.ndim != 2 or rec.shape[1] != 3:
            raise ValueError("rec_ijk must be (nrec, 3)")
        nsys = self._last_nsys
        E = np.empty((nsys, len(rec), 3), np.complex128) if e else None
        H = np.empty((nsys, len(rec), 3), np.complex128) if h else None
        self._check(self.lib.aphid_gpu_sweep_receivers(
            self._h, len(rec), rec.ctypes.data, E.ctypes.data if e else None,
            H.ctypes.data if h else None), "sweep_receivers")
        return E, H

    def sweep_time_apply(self, reps):
        """Launch the fused complex64 QMR pass `reps` times on the resident
        systems of the last mixed sweep (asynchronous; for timing; the
        solutions are not changed)."""
        self._check(self.lib.aphid_gpu_sweep_time_apply(self._h, int(reps)), "sweep_time_apply")

    def sweep_apply(self, x):
        """y = K x through the fused pass of the last batched sweep (complex64
        after mixed/auto, complex128 after fused64), for its system 0
        (testing hook: overwrites that sweep's inner vectors)."""
        x = np.ascontiguousarray(x, dtype=np.complex128).reshape(self.n)
        y = np.empty(self.n, np.complex128)
        self._check(self.lib.aphid_gpu_sweep_apply(self._h, x.ctypes.data, y.ctypes.data), "sweep_apply")
        return y

    def sweep_plane_kz(self):
        """z-planes per work item of the fused pass that ran last (the
        autotuner's choice unless plane_kz was fixed): the complex128 pass's
        after an escalating AUTO sweep or a FUSED64 sweep, else the complex64
        pass's; 0 before a mixed sweep."""
        return int(self.lib.aphid_gpu_sweep_plane_kz(self._h))

    def sweep_pass_config(self):
        """pipeline configuration of the complex64 pass in use (0: two load
        stages, two blocks per SM for model R; 1: three stages, one block)"""
        return int(self.lib.aphid_gpu_sweep_pass_config(self._h))

    def sweep_tile_shape(self):
        """plane-tile shape of the fused passes in use (0: 16 x 16 nodes,
        1: 32 x 8)"""
        return int(self.lib.aphid_gpu_sweep_tile_shape(self._h))

    def sweep_fetch(self, sys):
        x = np.empty(self.n, np.complex128)
        self._check(self.lib.aphid_gpu_sweep_fetch(self._h, int(sys), x.ctypes.data), "sweep_fetch")
        return x

    def gen_fields(self, omega, sol):
        """(B, E): B = curl A on faces [Bx|By|Bz], E on edges [Ex|Ey|Ez]."""
        nx, ny, nz = self.dims
        sol = _c128(sol, self.n)
        nb = [nx * (ny - 1) * (nz - 1), (nx - 1) * ny * (nz - 1), (nx - 1) * (ny - 1) * nz]
        B = np.empty(sum(nb), np.complex128)
        E = np.empty(self.off[3], np.complex128)
        bp = [B.ctypes.data, B.ctypes.data + 16 * nb[0], B.ctypes.data + 16 * (nb[0] + nb[1])]
        ep = [E.ctypes.data + 16 * o for o in self.off[:3]]
        self._check(self.lib.aphid_gpu_fields(self._h, float(omega), *self._blocks(sol), *bp,
                                              *ep), "gen_fields")
        return B, E


def sweep_group(jobs, precision="auto", target=1e-8, max_it=20000, inner_tol=0.0, max_outer=0,
                stall_window=0, fetch=True):
    """Sweeps of several meshes as one batched solve (aphid_gpu_sweep_group).

    jobs: list of (solver, omegas, sources, source_of_system) -- each solver
    a Solver bound to its own mesh and model, on the same device.  With
    precision "mixed" or "auto" and models of one kind, the complex64 passes
    of all meshes share one persistent launch per QMR iteration.  Returns a
    list of (X, infos) per job, as Solver.sweep returns them."""
    if not jobs:
        return []
    if precision not in PRECISIONS:
        raise AphidError("precision must be one of %s" % ", ".join(PRECISIONS))
    o = SweepOpts(PRECISIONS[precision], float(target), int(max_it), float(inner_tol), int(max_outer),
                  int(stall_window))
    arr = (GroupJob * len(jobs))()
    keep, outs = [], []
    for q, (sv, omegas, sources, sos) in enumerate(jobs):
        om = np.ascontiguousarray(np.atleast_1d(omegas), dtype=np.float64)
        nsys = om.size
        so = np.ascontiguousarray(np.arange(nsys) if sos is None else sos, dtype=np.int32)
        srcs, k = _sources(sources)
        X = np.empty((nsys, sv.n), np.complex128) if fetch else None
        infos = (Info * nsys)()
        keep += [om, so, srcs, k]
        outs.append((sv, X, infos, nsys))
        arr[q] = GroupJob(sv._h.value, nsys, om.ctypes.data, so.ctypes.data, len(sources),
                          C.cast(srcs, C.c_void_p).value, None, X.ctypes.data if X is not None else None,
                          C.cast(infos, C.c_void_p).value)
        sv._last_nsys = 0
    rc = load().aphid_gpu_sweep_group(len(jobs), arr, C.byref(o))
    if rc != APHID_OK:
        msgs = [load().aphid_gpu_last_error(sv._h).decode() for sv, _, _, _ in outs]
        raise AphidError("sweep_group: %s (%s)" % (ERRORS.get(rc, rc), "; ".join(m for m in msgs if m)))
    res = []
    for sv, X, infos, nsys in outs:
        sv._last_nsys = nsys
        res.append((X, [i.as_dict() for i in infos]))
    return res
