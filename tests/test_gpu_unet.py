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
