"""Host-side helpers of the learned initial guess (no GPU)."""
import numpy as np

from aphid_git_b200 import learn
from aphid_git_b200.abi import nunk


def test_pack_unpack_round_trip():
    dims = (7, 5, 4)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(nunk(*dims)) + 1j * rng.standard_normal(nunk(*dims))
    y = learn.pack_solution(x, dims)
    assert y.shape == (7 * 5 * 4, 8)
    g = learn.unpack_groups(y, dims)
    assert len(g) == 4
    assert np.abs(sum(g) - x).max() < 1e-6 * np.abs(x).max()
    # each group lives in its own block only
    nx, ny, nz = dims
    o = [0, (nx - 1) * ny * nz, (nx - 1) * ny * nz + nx * (ny - 1) * nz]
    assert np.all(g[1][:o[1]] == 0) and np.all(g[0][o[1]:] == 0)


def test_features_and_normalisation():
    dims = (6, 5, 4)
    sig = np.full((5, 4, 3), 1e-2)
    sig[:, :, 0] = 1e-8
    f = learn.features(sig, 10.0, [("+X", 3, 2, 2), ("-Y", 2, 3, 2)], dims)
    assert f.shape == (120, 3)
    assert np.allclose(f[:, 1], 0.25)
    assert f[:, 0].min() < 0 and np.isclose(f[:, 0].max(), 0.5)
    m = f[:, 2].reshape(4, 5, 6)
    assert m[1, 1, 2] == 1.0 and m[1, 1, 3] == 1.0          # +X edge (3,2,2)-(4,2,2), 1-based
    assert m[1, 1, 1] == -0.5 and m[1, 2, 1] == -0.5        # -Y edge (2,2,2)-(2,3,2)
    x = np.random.default_rng(1).standard_normal((50, 8)) * np.logspace(-6, 2, 50)[:, None]
    t = learn.compress(x)
    assert np.abs(t).max() <= 1.0 + 1e-6
    for g in range(4):
        m = np.sqrt(x[:, 2 * g] ** 2 + x[:, 2 * g + 1] ** 2).max()
        back = learn.expand(t[:, 2 * g:2 * g + 2]) * learn.EPS * m
        big = np.abs(x[:, 2 * g:2 * g + 2]) > 1e-3 * m
        assert np.allclose(back[big], x[:, 2 * g:2 * g + 2][big], rtol=1e-4)
