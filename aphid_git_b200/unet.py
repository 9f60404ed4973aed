"""Learned initial guess for the sweep: the host side of the 3-D U-Net.

The network maps (log10 sigma, log10 f, source mask) on the mesh nodes to
the eight real channels of (Ax, Ay, Az, Phi); its device kernels (tcgen05
BF16 GEMMs with FP32 accumulation under im2col convolutions) live in
libaphid_gpu.so behind include/aphid_unet.h.  The reference has no such
part: its QMR starts from zero (src/aphid_qmr.f90:230-233).  The network
only supplies x0, so it changes iteration counts and never the converged
answer.
"""
import ctypes as C

from . import abi

P = C.c_void_p
_bound = False


def lib():
    """The shared library with the U-Net entry points declared."""
    global _bound
    L = abi.load()
    if not _bound:
        L.aphid_unet_last_error.restype = C.c_char_p
        L.aphid_unet_gemm_bf16.argtypes = [P, C.c_int, P, C.c_int, P, C.c_int, P, C.c_int, C.c_int, C.c_int,
                                           C.c_int, C.c_int, P, P]
        _bound = True
    return L


def check(rc, what):
    if rc != 0:
        raise abi.AphidError("%s: %s" % (what, lib().aphid_unet_last_error().decode()))


def gemm_bf16(A, B, C_, bias=None, out=0, splitk=1, stream=None, err=None):
    """C_ (op)= A B^T for device tensors (torch: A, B bfloat16 row-major with
    K contiguous; C_ float32 or bfloat16).  out as in aphid_unet_gemm_bf16."""
    M, K = A.shape
    N = B.shape[0]
    check(lib().aphid_unet_gemm_bf16(A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), C_.data_ptr(),
                                     C_.stride(0), bias.data_ptr() if bias is not None else None, M, N, K, out,
                                     splitk, stream, err.data_ptr() if err is not None else None), "gemm_bf16")
