"""The allocation-free operator apply, for callers that cannot call cudaMalloc.

aphid_gpu_inprod_eps_noalloc serves code that runs inside a memory pool or a
framework allocator that owns all device memory, and hosts that must not
allocate once a run has started.  It takes only device pointers the caller
owns and keeps its scratch in a fixed array inside the library.  These tests
call it through the C ABI and check its output and its epsilon = in^T out
against the context entry point aphid_gpu_inprod_dev, on two calls in a row
with different inputs (the shared scratch keeps the previous call's contents,
so the second call shows that nothing stale leaks into the result).
Tolerances are those of the other complex128 operator tests: 1e-13 relative
(norm-wise) for the output, 1e-12 for epsilon, whose reduction order may differ.

Collected last (file name) so a run that stops at the first failure has
already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(rng, dims):
    from aphid_git_b200 import model
    from oracle import oracle as O
    xn, yn, zn = [np.cumsum(np.concatenate([[0.0], rng.uniform(50.0, 400.0, n - 1)]))
                  for n in dims]
    g = O.Grid(xn, yn, zn)
    cs = tuple(d - 1 for d in dims)
    sig_re = (10.0 ** rng.uniform(-4, 1, cs)).astype(np.float32)
    w = 2 * np.pi * 7.0
    k2 = O.gen_k2(g, model.sigma_hat("R", w, sig_re.ravel(order="F")), w)
    return (xn, yn, zn), g, k2


def test_noalloc_matches_context_apply_twice():
    import torch
    from aphid_git_b200 import Solver, model
    from aphid_git_b200.abi import inprod_eps_noalloc

    rng = np.random.default_rng(2024)
    dims = (37, 29, 23)
    (xn, yn, zn), g, k2 = _case(rng, dims)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)

    def to_dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    (dx, dxc), (dy, dyc), (dz, dzc) = model.spacings(xn), model.spacings(yn), model.spacings(zn)
    spacing = [to_dev(a) for a in (dx, dy, dz, dxc, dyc, dzc)]
    k2_d = to_dev(k2.view(np.float64))
    with Solver() as s:
        s.set_nodes(xn, yn, zn)
        for call in range(2):
            x = rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n)
            x_d = to_dev(x.view(np.float64))
            out_ref = torch.empty_like(x_d)
            out_new = torch.full_like(x_d, float("nan"))
            eps_ref = torch.zeros(2, dtype=torch.float64, device=dev)
            eps_new = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            s.inprod_dev(k2_d.data_ptr(), x_d.data_ptr(), out_ref.data_ptr(), eps_ref.data_ptr())
            torch.cuda.synchronize()
            rc = inprod_eps_noalloc(*dims, [t.data_ptr() for t in spacing], k2_d.data_ptr(),
                                    x_d.data_ptr(), out_new.data_ptr(), eps_new.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            assert rc == 0, (call, rc)
            a = out_new.cpu().numpy().view(np.complex128)
            b = out_ref.cpu().numpy().view(np.complex128)
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-13, call
            ea = complex(*eps_new.cpu().numpy())
            eb = complex(*eps_ref.cpu().numpy())
            assert abs(ea - eb) <= 1e-12 * abs(eb), (call, ea, eb)


def test_noalloc_rejects_meshes_beyond_its_scratch():
    import torch
    from aphid_git_b200.abi import NOALLOC_MAX_NODES, inprod_eps_noalloc
    p = torch.zeros(2, dtype=torch.float64, device="cuda").data_ptr()
    rc = inprod_eps_noalloc(NOALLOC_MAX_NODES + 1, 8, 8, [p] * 6, p, p, p, p, 0)
    assert rc == -1  # APHID_ERR_BADARG, before any device work
