"""The initial-guess network's device kernels against PyTorch FP32
references of the same operations (inputs rounded to BF16 first, so the
only difference left is the order of the FP32 accumulation)."""
import pytest

torch = pytest.importorskip("torch")
from aphid_git_b200 import unet

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float((a - b).norm() / b.norm().clamp_min(1e-30))


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (256, 96, 192), (384, 128, 448), (128, 256, 64)])
def test_gemm_matches_fp32(M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    bias = torch.randn(N, device="cuda", generator=g)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ref = A.float() @ B.float().T
    C = torch.empty(M, N, device="cuda")
    unet.gemm_bf16(A, B, C, err=err)
    torch.cuda.synchronize()
    assert int(err) == 0
    assert rel(C, ref) < 1e-5
    unet.gemm_bf16(A, B, C, bias=bias)
    assert rel(C, ref + bias) < 1e-5
    Cb = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    unet.gemm_bf16(A, B, Cb, bias=bias, out=1)
    assert rel(Cb.float(), torch.relu(ref + bias)) < 1e-2
    unet.gemm_bf16(A, B, Cb, bias=bias, out=2)
    assert rel(Cb.float(), ref + bias) < 1e-2
    # split-K accumulation into an existing C
    C0 = torch.randn(M, N, device="cuda", generator=g)
    C1 = C0.clone()
    unet.gemm_bf16(A, B, C1, out=3, splitk=3)
    torch.cuda.synchronize()
    assert rel(C1 - C0, ref) < 1e-5


def test_gemm_strided_operands():
    """Leading dimensions larger than K (sub-blocks of bigger buffers)."""
    g = torch.Generator(device="cuda").manual_seed(7)
    Abig = torch.randn(256, 200, device="cuda", generator=g).bfloat16()
    Bbig = torch.randn(64, 136, device="cuda", generator=g).bfloat16()
    A, B = Abig[:, :128], Bbig[:, :128]
    C = torch.zeros(256, 80, device="cuda")
    unet.gemm_bf16(A, B, C[:, :64])
    ref = A.float() @ B.float().T
    assert rel(C[:, :64], ref) < 1e-5
    assert float(C[:, 64:].abs().max()) == 0.0


def test_gemm_rejects_bad_shapes():
    A = torch.zeros(100, 64, device="cuda", dtype=torch.bfloat16)
    B = torch.zeros(16, 64, device="cuda", dtype=torch.bfloat16)
    C = torch.zeros(100, 16, device="cuda")
    with pytest.raises(Exception):
        unet.gemm_bf16(A, B, C)


def _ref_case(dims, seed):
    import numpy as np
    from oracle import unet_ref as R
    rng = np.random.default_rng(seed)
    X, Y, Z = dims
    Xp, Yp, Zp = R.padded(dims)
    p = (R.init_params(seed) * 0.7).astype(np.float32)
    x = rng.standard_normal((X * Y * Z, 3)).astype(np.float32)
    t = rng.standard_normal((X * Y * Z, 8)).astype(np.float32)
    w = (rng.random(X * Y * Z) > 0.3).astype(np.float32)
    # the same case on the padded volume for the reference
    def pad(a):
        c = a.shape[1]
        out = np.zeros((Zp, Yp, Xp, c))
        out[:Z, :Y, :X] = a.reshape(Z, Y, X, c)
        return out.reshape(-1, c)
    wp = pad(w[:, None])[:, 0]
    return p, x, t, w, pad(x), pad(t), wp, (Xp, Yp, Zp)


def test_network_forward_and_gradients_match_cpu_reference():
    """The whole network, forward and back-propagation, against the CPU
    restatement with the same BF16 rounding points (oracle/unet_ref.py) on a
    ragged 30 x 27 x 22 volume (padded to 32 x 32 x 24).  Tolerance: per
    layer, the parameter gradient may differ from the restatement's by at
    most twice the restatement's own BF16 rounding noise (its distance from
    the same computation in FP64): rounding ties resolved in a different
    accumulation order flip ReLU masks and BF16 roundings, and the deep
    layers see few voxels."""
    import numpy as np
    from oracle import unet_ref as R
    dims = (30, 27, 22)
    p, x, t, w, xp, tp, wp, pd = _ref_case(dims, 5)
    X, Y, Z = dims
    y_ref, st = R.forward(p.astype(np.float64), xp, pd)
    loss_ref, dy = R.loss_grad(y_ref, tp, wp)
    g_ref = R.backward(dy, st)
    y64, st64 = R.forward(p.astype(np.float64), xp, pd, bf=False)
    g64 = R.backward(R.loss_grad(y64, tp, wp)[1], st64, bf=False)
    y_ref = y_ref.reshape(pd[2], pd[1], pd[0], 8)[:Z, :Y, :X].reshape(-1, 8)
    with unet.UNet(*dims, train=True) as net:
        net.set_params(p)
        xd = torch.from_numpy(x).cuda()
        yd = torch.empty(X * Y * Z, 8, device="cuda")
        net.forward(xd, yd)
        y = yd.cpu().numpy()
        assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < 1e-2
        loss = net.train_step(xd, torch.from_numpy(t).cuda(), torch.from_numpy(w).cuda(), update=False)
        g = net.grads()
    assert abs(loss - loss_ref) < 1e-3 * loss_ref
    o = 0
    for ci, co in R.LAYERS:
        n = 27 * ci * co + co
        a, b, c = g[o:o + n], g_ref[o:o + n], g64[o:o + n]
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        noise = np.linalg.norm(b - c) / np.linalg.norm(c)
        assert err <= 2 * noise + 1e-3, ((ci, co), err, noise)
        o += n


def test_training_reduces_the_loss():
    import numpy as np
    dims = (16, 16, 12)
    X, Y, Z = dims
    rng = np.random.default_rng(2)
    x = rng.standard_normal((X * Y * Z, 3)).astype(np.float32)
    # a smooth target that depends on the inputs
    t = np.tanh(np.concatenate([x, x[:, :2] * x[:, 2:3], x * 0.5], axis=1)[:, :8]).astype(np.float32)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    with unet.UNet(*dims, train=True, seed=3) as net:
        l0 = net.train_step(xd, td, lr=1e-3)
        for _ in range(60):
            l1 = net.train_step(xd, td, lr=1e-3)
    assert l1 < 0.5 * l0, (l0, l1)
