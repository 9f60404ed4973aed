"""The CPU restatement of the initial-guess network checks itself: its
backward pass against central finite differences of its forward pass (FP64,
no BF16 rounding), on a volume of 8^3 nodes (three poolings down to one)."""
import numpy as np

from oracle import unet_ref as R


def test_param_count_matches_architecture():
    # 4 levels, 16/32/64/128 channels, 3^3 kernels, 3 inputs, 8 outputs
    assert R.param_count() == sum(27 * a * b + b for a, b in R.LAYERS)
    assert [co for _, co in R.ENC] == [16, 16, 32, 32, 64, 64, 128, 128]
    assert R.HEAD == (16, 8)


def test_backward_matches_finite_differences():
    dims = (8, 8, 8)
    rng = np.random.default_rng(1)
    p = R.init_params(3) * 0.5
    x = rng.standard_normal((512, 3))
    t = rng.standard_normal((512, 8))
    w = (rng.random(512) > 0.2).astype(float)

    def L(pp):
        y, _ = R.forward(pp, x, dims, bf=False)
        return R.loss_grad(y, t, w)[0]

    y, st = R.forward(p, x, dims, bf=False)
    _, dy = R.loss_grad(y, t, w)
    g = R.backward(dy, st, bf=False)
    assert g.shape == p.shape
    # a few weights and biases of every layer
    o, idx = 0, []
    for ci, co in R.LAYERS:
        nW = 27 * ci * co
        idx += list(o + rng.choice(nW, 2, replace=False)) + [o + nW + int(rng.integers(co))]
        o += nW + co
    h = 1e-6  # small enough that no ReLU changes state inside the step
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (L(p + e) - L(p - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 65504.0], np.float32)
    r = R.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0           # tie to even
    assert r[2] == 1.0 + 2 ** -7
    assert abs(r[3] + 3.140625) < 1e-12
