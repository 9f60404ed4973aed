"""The allocation-free operator apply, for callers that cannot call cudaMalloc.

aphid_gpu_inprod_eps_noalloc serves code that runs inside a memory pool or a
framework allocator that owns all device memory, and hosts that must not
allocate once a run has started.  It takes only device pointers the caller
owns and keeps its scratch in a fixed array inside the library.  These tests
call it through the C ABI and check its output and its epsilon = in^T out
against the context entry point aphid_gpu_inprod_dev and against the CPU
oracle's inprod, on two calls in a row with different inputs (the shared
scratch keeps the previous call's contents, so the second call shows that
nothing stale leaks into the result).  A second case runs a mesh at the
1024-node edge whose column count forces z-slabs deeper than 32 planes, the
tiling that keeps the partial sums within the fixed slots.
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
    from oracle import oracle as O

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
            # and against the oracle's operator (src/aphid.f90 inprod_x/y/z/p)
            o = O.inprod(g, k2, x)
            assert np.linalg.norm(a - o) / np.linalg.norm(o) < 1e-13, call
            eo = complex(np.sum(x * o))
            assert abs(ea - eo) <= 1e-12 * abs(eo), (call, ea, eo)


def test_noalloc_deep_slabs_at_the_node_limit():
    # 65 x 1024 x 683 nodes: 3 x 256 tile columns of 32 x 4 nodes over 683
    # planes need z-slabs of 33 planes to fit 16384 partial-sum slots
    # (181 M unknowns, about 41 GB on the device with the context path)
    import torch
    from aphid_git_b200 import Solver, model
    from aphid_git_b200.abi import NOALLOC_MAX_NODES, NOALLOC_MAX_SLOTS, inprod_eps_noalloc

    dims = (65, NOALLOC_MAX_NODES, 683)
    cols = -(-dims[0] // 32) * -(-dims[1] // 4)
    assert cols * dims[2] > 32 * NOALLOC_MAX_SLOTS  # beyond 32-plane slabs
    rng = np.random.default_rng(77)
    xn, yn, zn = [np.cumsum(np.concatenate([[0.0], rng.uniform(50.0, 400.0, n - 1)])) for n in dims]
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    (dx, dxc), (dy, dyc), (dz, dzc) = model.spacings(xn), model.spacings(yn), model.spacings(zn)
    spacing = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (dx, dy, dz, dxc, dyc, dzc)]
    with Solver() as s:
        s.set_nodes(xn, yn, zn)
        gen = torch.Generator(device=dev).manual_seed(5)
        k2_d = torch.randn(2 * s.n, dtype=torch.float64, device=dev, generator=gen)
        x_d = torch.randn(2 * s.n, dtype=torch.float64, device=dev, generator=gen)
        out_ref = torch.empty_like(x_d)
        out_new = torch.full_like(x_d, float("nan"))
        eps_ref = torch.zeros(2, dtype=torch.float64, device=dev)
        eps_new = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
        # the context path runs on its own non-blocking stream: torch's fills
        # of the inputs and of eps_ref must have landed before it starts
        torch.cuda.synchronize()
        s.inprod_dev(k2_d.data_ptr(), x_d.data_ptr(), out_ref.data_ptr(), eps_ref.data_ptr())
        torch.cuda.synchronize()
        rc = inprod_eps_noalloc(*dims, [t.data_ptr() for t in spacing], k2_d.data_ptr(), x_d.data_ptr(),
                                out_new.data_ptr(), eps_new.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert rc == 0, rc
        rel = float(torch.linalg.vector_norm(out_new - out_ref) / torch.linalg.vector_norm(out_ref))
        assert rel < 1e-13, rel
        ea, eb = complex(*eps_new.cpu().numpy()), complex(*eps_ref.cpu().numpy())
        assert abs(ea - eb) <= 1e-12 * abs(eb), (ea, eb)
        del k2_d, x_d, out_ref, out_new
    torch.cuda.empty_cache()


def test_noalloc_rejects_meshes_beyond_its_scratch():
    import torch
    from aphid_git_b200.abi import NOALLOC_MAX_NODES, inprod_eps_noalloc
    p = torch.zeros(2, dtype=torch.float64, device="cuda").data_ptr()
    rc = inprod_eps_noalloc(NOALLOC_MAX_NODES + 1, 8, 8, [p] * 6, p, p, p, p, 0)
    assert rc == -1  # APHID_ERR_BADARG, before any device work
