"""Learned initial guess for the QMR solve (no counterpart in the reference,
whose QMR starts from zero, src/aphid_qmr.f90:230-233).

A 3-D U-Net (aphid_git_b200/unet.py; device kernels in
csrc/aphid_unet.cu) maps, on the mesh nodes,

    (log10 sigma, log10 f, source mask)  ->  (Re, Im) of (Ax, Ay, Az, Phi)

each real channel compressed as asinh(x / (EPS peak)) / asinh(1 / EPS),
peak the field's largest magnitude: the fields span many decades between
the source and the far edge, and in this form a network error is a
relative error at every magnitude.  The amplitudes are then fitted by least
squares: x0 = sum_g alpha_g x_g with
complex alpha minimising ||b - K x0||_2 (four operator applies and a 4 x 4
solve), so x0 never has a larger residual than the zero start.  The guess
enters the sweep (or aphid_gpu_qmr) as x0 and changes iteration counts, never
the converged answer; without weights the solve starts from zero.

Training data are solutions of the solver itself (the mixed sweep to a true
FP64 residual of 1e-8).  Command line:

    python -m aphid_git_b200.learn train --models 100 --freqs 20 --out W.npz
    python -m aphid_git_b200.learn eval  --weights W.npz --seeds 901 902
"""
import argparse
import json
import os
import time

import numpy as np

from . import model
from .abi import Solver

HERE = os.path.dirname(os.path.abspath(__file__))
PRETRAINED = os.path.join(HERE, "weights", "unet_train64.npz")
FMIN, FMAX = 1e-3, 1e4   # the reference's Jacobi-QMR converges up to about 1e4 Hz on these meshes
EPS = 1e-5               # smallest magnitude (relative to the peak) the compression resolves
# A guess is used only when its fitted residual is below this fraction of
# ||b||.  Per-node errors of a few percent already leave the residual at
# ||b|| and cost iterations (measured on a 40^3 heterogeneous mesh: white
# errors of 2% in the compressed form gave 710 iterations against 699 from
# zero; smooth 1% errors gave 510-600), so a poor guess is dropped.
ACCEPT = 0.5
_ASINH = float(np.arcsinh(1.0 / EPS))


# ------------------------------------------------------------------ features
def node_log_sigma(sig_cells):
    """log10 of the cell conductivity averaged onto the nodes (the up to 8
    cells around each node), [nz][ny][nx]."""
    ls = np.log10(np.asarray(sig_cells, np.float64))          # (cx, cy, cz)
    p = np.pad(ls, 1, mode="edge")                              # (cx+2, ...)
    acc = np.zeros((ls.shape[0] + 1, ls.shape[1] + 1, ls.shape[2] + 1))
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                acc += p[a:a + ls.shape[0] + 1, b:b + ls.shape[1] + 1, c:c + ls.shape[2] + 1]
    return (acc / 8.0).transpose(2, 1, 0)                       # (nz, ny, nx)


def features(sig_cells, freq, dipoles, dims):
    """[V][3] float32: (log10 sigma + 4) / 4, log10 f / 4, source mask
    (+-1 at the two end nodes of each x-dipole, +-0.5 for y, +-0.25 for z)."""
    nx, ny, nz = dims
    f = np.zeros((nz, ny, nx, 3), np.float32)
    f[..., 0] = (node_log_sigma(sig_cells) + 4.0) / 4.0
    f[..., 1] = np.log10(freq) / 4.0
    val = {"X": 1.0, "Y": 0.5, "Z": 0.25}
    for d, i, j, k in dipoles:
        s = (1.0 if d[0] == "+" else -1.0) * val[d[1]]
        t = [i - 1, j - 1, k - 1]
        if d[0] == "-":
            t["XYZ".index(d[1])] -= 1
        h = list(t)
        h["XYZ".index(d[1])] += 1
        for q in (t, h):
            if 0 <= q[0] < nx and 0 <= q[1] < ny and 0 <= q[2] < nz:
                f[q[2], q[1], q[0], 2] += s
    return f.reshape(-1, 3)


def _blocks(dims):
    nx, ny, nz = dims
    return [(nx - 1, ny, nz), (nx, ny - 1, nz), (nx, ny, nz - 1), (nx, ny, nz)]


def pack_solution(x, dims):
    """reference-layout [Ax|Ay|Az|Phi] -> [V][8] on the nodes (each edge on
    its lower end node)."""
    nx, ny, nz = dims
    out = np.zeros((nz, ny, nx, 8), np.float32)
    o = 0
    for g, (a, b, c) in enumerate(_blocks(dims)):
        blk = x[o:o + a * b * c].reshape((a, b, c), order="F").transpose(2, 1, 0)
        out[:c, :b, :a, 2 * g] = blk.real
        out[:c, :b, :a, 2 * g + 1] = blk.imag
        o += a * b * c
    return out.reshape(-1, 8)


def unpack_groups(y, dims):
    """[V][8] on the nodes -> four reference-layout vectors, one per field
    (Ax, Ay, Az, Phi), each zero outside its own block."""
    nx, ny, nz = dims
    t = y.reshape(nz, ny, nx, 8)
    n = sum(a * b * c for a, b, c in _blocks(dims))
    out, o = [], 0
    for g, (a, b, c) in enumerate(_blocks(dims)):
        v = np.zeros(n, np.complex128)
        blk = t[:c, :b, :a, 2 * g] + 1j * t[:c, :b, :a, 2 * g + 1]
        v[o:o + a * b * c] = blk.transpose(2, 1, 0).reshape(-1, order="F")
        out.append(v)
        o += a * b * c
    return out


def compress(t):
    """per field (channel pair): asinh(x / (EPS peak)) / asinh(1 / EPS)"""
    t = np.asarray(t, np.float64).copy()
    for g in range(4):
        m = np.sqrt(t[:, 2 * g] ** 2 + t[:, 2 * g + 1] ** 2).max()
        if m > 0:
            t[:, 2 * g:2 * g + 2] = np.arcsinh(t[:, 2 * g:2 * g + 2] / (EPS * m)) / _ASINH
    return t.astype(np.float32)


def expand(y):
    """the inverse of compress up to one scale per field (fitted later)"""
    return np.sinh(np.clip(np.asarray(y, np.float64), -1.5, 1.5) * _ASINH)


def fit_amplitudes(solver, k2, b, groups):
    """x0 = sum_g alpha_g x_g minimising ||b - K x0||_2 (complex alpha)."""
    kx = [solver.inprod(k2, g) for g in groups]
    G = np.array([[np.vdot(a, c) for c in kx] for a in kx])
    r = np.array([np.vdot(a, b) for a in kx])
    alpha = np.linalg.lstsq(G, r, rcond=None)[0]
    return sum(a * g for a, g in zip(alpha, groups)), alpha


# ---------------------------------------------------------------- inference
class Guess:
    """Initial guesses from trained parameters for one mesh (any size)."""

    def __init__(self, params, dims):
        import torch
        from . import unet
        self.torch = torch
        self.dims = dims
        self.net = unet.UNet(*dims, train=False)
        self.net.set_params(params)

    def predict(self, sig_cells, freq, dipoles):
        torch = self.torch
        x = torch.from_numpy(features(sig_cells, freq, dipoles, self.dims)).cuda()
        y = torch.empty(x.shape[0], 8, device="cuda")
        self.net.forward(x, y)
        return y.cpu().numpy()

    def x0(self, solver, sig_cells, freq, dipoles, accept=ACCEPT):
        """(initial guess or None, its relative residual) for one system:
        the fitted guess when its residual ||b - K x0|| / ||b|| is below
        `accept`, else None (the solve starts from zero)"""
        w = 2 * np.pi * freq
        k2 = solver.gen_k2(model.sigma_hat("R", w, np.asarray(sig_cells).ravel(order="F")), w)
        b, _ = model.gen_rhs(solver.xn, solver.yn, solver.zn, 5, dipoles)
        groups = unpack_groups(expand(self.predict(sig_cells, freq, dipoles)), self.dims)
        x0 = fit_amplitudes(solver, k2, b, groups)[0]
        r0 = float(np.linalg.norm(b - solver.inprod(k2, x0)) / np.linalg.norm(b))
        return (x0 if r0 < accept else None), r0

    def close(self):
        self.net.close()


def load_params(path=None):
    """trained parameters (FP32), or None when there are none: the solve then
    starts from zero"""
    path = path or PRETRAINED
    if not os.path.exists(path):
        return None
    return np.load(path)["params"].astype(np.float32)


# ----------------------------------------------------------------- training
def generate(seeds, nfreq, rng, max_it=8000, verbose=True):
    """(features, compressed targets) of converged mixed-sweep solutions of
    the train64 generator, nfreq log-uniform frequencies per model."""
    data = []
    for s in seeds:
        m = model.make_model("train64", seed=int(s))
        dims = m.dims
        freqs = np.exp(rng.uniform(np.log(FMIN), np.log(FMAX), nfreq))
        with Solver() as sol:
            sol.set_nodes(m.xn, m.yn, m.zn)
            sol.set_model("R", m.sig_re)
            X, infos = sol.sweep([2 * np.pi * f for f in freqs], m.sources, [0] * nfreq, precision="mixed",
                                 target=1e-8, max_it=max_it)
        kept = 0
        for q, f in enumerate(freqs):
            if infos[q]["status_name"] != "converged":
                continue
            data.append((features(m.sig_re, f, m.sources[0], dims), compress(pack_solution(X[q], dims))))
            kept += 1
        if verbose:
            print("model %d: %d of %d systems converged" % (s, kept, nfreq), flush=True)
    return data, dims


def train(data, dims, epochs, lr=1e-3, seed=0, verbose=True):
    import torch
    from . import unet
    rng = np.random.default_rng(seed)
    xs = [torch.from_numpy(a).cuda() for a, _ in data]
    ts = [torch.from_numpy(b).cuda() for _, b in data]
    hist = []
    with unet.UNet(*dims, train=True, seed=seed) as net:
        steps, k = epochs * len(data), 0
        for ep in range(epochs):
            tot = 0.0
            for i in rng.permutation(len(data)):
                lr_k = lr * 0.5 * (1 + np.cos(np.pi * k / steps)) + 1e-5
                tot += net.train_step(xs[i], ts[i], lr=lr_k)
                k += 1
            hist.append(tot / len(data))
            if verbose:
                print("epoch %d loss %.4e" % (ep, hist[-1]), flush=True)
        return net.params(), hist


# --------------------------------------------------------------- evaluation
def evaluate(params, seeds, freqs, config="eval160", max_it=20000, verbose=True):
    """complex128 QMR iterations to 1e-8 (the reference's recurrence) from
    zero and from the learned guess, per (seed, frequency)"""
    rows = []
    for s in seeds:
        m = model.make_model(config, seed=int(s))
        with Solver() as sol:
            sol.set_nodes(m.xn, m.yn, m.zn)
            g = Guess(params, m.dims)
            for f in freqs:
                w = 2 * np.pi * f
                k2 = sol.gen_k2(model.sigma_hat("R", w, m.sig_re.ravel(order="F")), w)
                dg = sol.gen_diag(k2)
                b, _ = model.gen_rhs(m.xn, m.yn, m.zn, 5, m.sources[0])
                t0 = time.time()
                x0, r0 = g.x0(sol, m.sig_re, f, m.sources[0])
                tg = time.time() - t0
                _, i_zero, _ = sol.qmr(k2, dg, b, 1e-8, max_it)
                _, i_nn, _ = sol.qmr(k2, dg, b, 1e-8, max_it, x0=x0)
                row = {"seed": int(s), "freq": float(f), "iters_zero": i_zero["iters"], "iters_learned": i_nn["iters"],
                       "rel_resid_x0": r0, "guess_used": x0 is not None, "guess_s": tg,
                       "status_learned": i_nn["status_name"]}
                rows.append(row)
                if verbose:
                    print(json.dumps(row), flush=True)
            g.close()
    return rows


def conv_flops(dims):
    """FLOPs of one forward pass (the GEMMs of the 15 convolutions)"""
    from . import unet  # noqa: F401  (same layer list as the device code)
    layers = [(3, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 128, 3),
              (128, 128, 3), (192, 64, 2), (64, 64, 2), (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0),
              (16, 8, 0)]
    v0 = np.prod([-(-d // 8) * 8 for d in dims])
    return sum(2.0 * v0 / 8 ** lev * 27 * ci * co for ci, co, lev in layers)


def speed(dims, steps):
    """ms per training step and per forward pass, and the GEMM FLOP rate
    (backward = twice the forward FLOPs: dW and dCol)"""
    import torch
    from . import unet
    rng = np.random.default_rng(0)
    V = int(np.prod(dims))
    x = torch.from_numpy(rng.standard_normal((V, 3)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((V, 8)).astype(np.float32) * 0.1).cuda()
    y = torch.empty(V, 8, device="cuda")
    out = {"dims": list(dims), "forward_gflop": conv_flops(dims) / 1e9}
    with unet.UNet(*dims, train=True) as net:
        for _ in range(3):
            net.train_step(x, t, lr=1e-4)
        torch.cuda.synchronize()
        t0 = time.time()
        for _ in range(steps):
            net.train_step(x, t, lr=1e-4)
        torch.cuda.synchronize()
        out["train_step_ms"] = (time.time() - t0) / steps * 1e3
        for _ in range(3):
            net.forward(x, y)
        torch.cuda.synchronize()
        t0 = time.time()
        for _ in range(steps):
            net.forward(x, y)
        torch.cuda.synchronize()
        out["forward_ms"] = (time.time() - t0) / steps * 1e3
    out["train_tflops"] = 3 * out["forward_gflop"] / out["train_step_ms"]
    out["forward_tflops"] = out["forward_gflop"] / out["forward_ms"]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--models", type=int, default=100)
    t.add_argument("--freqs", type=int, default=20)
    t.add_argument("--epochs", type=int, default=10)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--first-seed", type=int, default=1000)
    t.add_argument("--out", default=PRETRAINED)
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=PRETRAINED)
    e.add_argument("--config", default="eval160")
    e.add_argument("--seeds", type=int, nargs="+", default=[901, 902])
    e.add_argument("--freqs", type=float, nargs="+", default=[1e-2, 1.0, 1e2])
    sp = sub.add_parser("speed")
    sp.add_argument("--dims", type=int, nargs=3, default=[65, 65, 49])
    sp.add_argument("--steps", type=int, default=20)
    a = ap.parse_args(argv)
    if a.cmd == "speed":
        print(json.dumps(speed(tuple(a.dims), a.steps)))
        return
    if a.cmd == "train":
        rng = np.random.default_rng(a.first_seed)
        t0 = time.time()
        data, dims = generate(range(a.first_seed, a.first_seed + a.models), a.freqs, rng)
        t1 = time.time()
        params, hist = train(data, dims, a.epochs, lr=a.lr)
        t2 = time.time()
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        np.savez_compressed(a.out, params=params.astype(np.float16),
                            meta=json.dumps({"models": a.models, "freqs": a.freqs, "epochs": a.epochs,
                                             "samples": len(data), "loss": hist, "config": "train64",
                                             "fmin": FMIN, "fmax": FMAX, "first_seed": a.first_seed}))
        print(json.dumps({"samples": len(data), "data_s": t1 - t0, "train_s": t2 - t1, "loss": hist[-1],
                          "out": a.out}))
    else:
        p = load_params(a.weights)
        if p is None:
            raise SystemExit("no weights at %s" % a.weights)
        evaluate(p, a.seeds, a.freqs, a.config)


if __name__ == "__main__":
    main()
