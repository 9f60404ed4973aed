"""CPU restatement of the initial-guess network (test infrastructure only:
the tests use it to check the device kernels; nothing in the product
imports it).

The network has no counterpart in the reference (its QMR starts from zero,
src/aphid_qmr.f90:230-233).  This module fixes its semantics for the
device implementation (aphid_git_b200/csrc/aphid_unet.cu):

  volume   nodes (X, Y, Z) padded to multiples of 8; voxel v = x + Xp (y + Yp z);
           activations [V][C], channels last
  conv     3x3x3, zero padding ("same"), weights W[co][tap*Cin + ci] with
           tap = ((dz+1)*3 + (dy+1))*3 + (dx+1), bias b[co]
  layers   enc: 3->16, 16->16 | pool | 16->32, 32->32 | pool | 32->64, 64->64
           | pool | 64->128, 128->128 ; dec: up(128) ++ skip(64) -> 64, 64->64 ;
           up(64) ++ skip(32) -> 32, 32->32 ; up(32) ++ skip(16) -> 16, 16->16 ;
           head 16->8 (no ReLU).  pool = 2x2x2 mean, up = nearest x2.
  rounding BF16 (round to nearest even) for weights, stored activations and
           the GEMM operands of the backward pass; FP32/FP64 elsewhere.

With bf16=False everything is FP64: used to finite-difference the
backward formulas themselves.
"""
import numpy as np

ENC = [(3, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128)]
DEC = [(192, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16)]
HEAD = (16, 8)
LAYERS = ENC + DEC + [HEAD]


def param_count():
    return sum(27 * ci * co + co for ci, co in LAYERS)


def unpack(params):
    """flat parameter vector -> [(W [co][27 ci], b [co])]"""
    out, o = [], 0
    for ci, co in LAYERS:
        W = params[o:o + 27 * ci * co].reshape(co, 27 * ci)
        o += 27 * ci * co
        b = params[o:o + co]
        o += co
        out.append((W, b))
    return out


def init_params(seed):
    """He-normal weights, zero biases (the device initialiser draws its own
    numbers; this one serves the tests)."""
    rng = np.random.default_rng(seed)
    ps = []
    for ci, co in LAYERS:
        ps.append(rng.standard_normal(27 * ci * co) * np.sqrt(2.0 / (27 * ci)))
        ps.append(np.zeros(co))
    return np.concatenate(ps)


def bf16(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def padded(dims):
    return tuple(-(-d // 8) * 8 for d in dims)


def _taps():
    return [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def im2col(a, dims):
    X, Y, Z = dims
    C = a.shape[1]
    t = a.reshape(Z, Y, X, C)
    p = np.zeros((Z + 2, Y + 2, X + 2, C))
    p[1:-1, 1:-1, 1:-1] = t
    cols = [p[1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X].reshape(-1, C) for dx, dy, dz in _taps()]
    return np.concatenate(cols, axis=1)


def col2im(dc, dims, C):
    X, Y, Z = dims
    p = np.zeros((Z + 2, Y + 2, X + 2, C))
    for t, (dx, dy, dz) in enumerate(_taps()):
        p[1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X] += dc[:, t * C:(t + 1) * C].reshape(Z, Y, X, C)
    return p[1:-1, 1:-1, 1:-1].reshape(-1, C)


def pool(a, dims):
    X, Y, Z = dims
    C = a.shape[1]
    t = a.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C)
    return t.mean(axis=(1, 3, 5)).reshape(-1, C)


def pool_back(g, dims):
    X, Y, Z = dims
    C = g.shape[1]
    t = g.reshape(Z // 2, 1, Y // 2, 1, X // 2, 1, C) / 8.0
    return np.broadcast_to(t, (Z // 2, 2, Y // 2, 2, X // 2, 2, C)).reshape(-1, C)


def up(a, dims):  # dims: the fine volume
    X, Y, Z = dims
    C = a.shape[1]
    t = a.reshape(Z // 2, 1, Y // 2, 1, X // 2, 1, C)
    return np.broadcast_to(t, (Z // 2, 2, Y // 2, 2, X // 2, 2, C)).reshape(-1, C)


def up_back(g, dims):
    X, Y, Z = dims
    C = g.shape[1]
    return g.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(1, 3, 5)).reshape(-1, C)


def forward(params, x, dims, bf=True):
    """x: [V][3] input features on the padded volume; returns (y [V][8],
    cache for backward)."""
    R = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    P = [(R(W), np.asarray(b, np.float64)) for W, b in unpack(params)]
    d1 = tuple(dims)
    d2 = tuple(d // 2 for d in d1)
    d3 = tuple(d // 2 for d in d2)
    d4 = tuple(d // 2 for d in d3)
    cache = []

    def conv(a, d, li, relu=True):
        col = im2col(a, d)
        z = col @ P[li][0].T + P[li][1]
        out = R(np.maximum(z, 0.0)) if relu else z
        cache.append((li, col, out, d, a.shape[1], relu))
        return out

    a = R(x)
    a = conv(a, d1, 0)
    s1 = conv(a, d1, 1)
    a = R(pool(s1, d1))
    a = conv(a, d2, 2)
    s2 = conv(a, d2, 3)
    a = R(pool(s2, d2))
    a = conv(a, d3, 4)
    s3 = conv(a, d3, 5)
    a = R(pool(s3, d3))
    a = conv(a, d4, 6)
    a = conv(a, d4, 7)
    a = np.concatenate([up(a, d3), s3], axis=1)
    a = conv(a, d3, 8)
    a = conv(a, d3, 9)
    a = np.concatenate([up(a, d2), s2], axis=1)
    a = conv(a, d2, 10)
    a = conv(a, d2, 11)
    a = np.concatenate([up(a, d1), s1], axis=1)
    a = conv(a, d1, 12)
    a = conv(a, d1, 13)
    y = conv(a, d1, 14, relu=False)
    return y, (P, cache, (d1, d2, d3, d4))


def loss_grad(y, target, weight):
    """mean weighted squared error over the 8 channels and its gradient"""
    w = weight[:, None] * np.ones((1, 8))
    r = y - target
    den = max(w.sum(), 1e-30)
    return float((w * r * r).sum() / den), 2.0 * w * r / den


def backward(dy, state, bf=True):
    """Parameter gradients (flat, the layout of the parameters) for dL/dy."""
    R = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    P, cache, (d1, d2, d3, d4) = state
    grads = [None] * len(LAYERS)
    by_layer = {c[0]: c for c in cache}

    def conv_back(li, g):
        _, col, out, d, cin, relu = by_layer[li]
        dz = g * (out > 0) if relu else g
        dzb = R(dz)
        grads[li] = (dzb.T @ col, dz.sum(axis=0))
        return col2im(dzb @ P[li][0], d, cin)

    g = conv_back(14, dy)
    g = conv_back(13, g)
    g = conv_back(12, g)           # [V1][48] = up(32) ++ s1(16)
    g_s1 = g[:, 32:]
    g = up_back(g[:, :32], d1)
    g = conv_back(11, g)
    g = conv_back(10, g)           # [V2][96] = up(64) ++ s2(32)
    g_s2 = g[:, 64:]
    g = up_back(g[:, :64], d2)
    g = conv_back(9, g)
    g = conv_back(8, g)            # [V3][192] = up(128) ++ s3(64)
    g_s3 = g[:, 128:]
    g = up_back(g[:, :128], d3)
    g = conv_back(7, g)
    g = conv_back(6, g)
    g = pool_back(g, d3) + g_s3
    g = conv_back(5, g)
    g = conv_back(4, g)
    g = pool_back(g, d2) + g_s2
    g = conv_back(3, g)
    g = conv_back(2, g)
    g = pool_back(g, d1) + g_s1
    g = conv_back(1, g)
    conv_back(0, g)
    return np.concatenate([np.concatenate([dw.ravel(), db]) for dw, db in grads])
