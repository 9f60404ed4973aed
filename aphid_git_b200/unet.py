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


def _bind_net(L):
    L.aphid_unet_param_count.restype = C.c_longlong
    L.aphid_unet_create.argtypes = [C.POINTER(P), C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong]
    L.aphid_unet_destroy.argtypes = [P]
    L.aphid_unet_get_params.argtypes = [P, P]
    L.aphid_unet_set_params.argtypes = [P, P]
    L.aphid_unet_forward.argtypes = [P, P, P, P]
    L.aphid_unet_train_step.argtypes = [P, P, P, P, C.c_float, C.c_int, C.POINTER(C.c_double), P]
    L.aphid_unet_get_grads.argtypes = [P, P]


class UNet:
    """One network object: buffers for a volume of X x Y x Z nodes (device
    tensors in and out, torch for the plumbing).  Parameters move between
    objects through params / set_params (FP32 host arrays)."""

    def __init__(self, X, Y, Z, train=False, seed=0):
        import numpy as np
        self.np = np
        self.L = lib()
        _bind_net(self.L)
        self.dims = (X, Y, Z)
        self._h = P()
        check(self.L.aphid_unet_create(C.byref(self._h), X, Y, Z, int(train), seed), "unet_create")

    @staticmethod
    def param_count():
        L = lib()
        _bind_net(L)
        return int(L.aphid_unet_param_count())

    def close(self):
        if self._h:
            self.L.aphid_unet_destroy(self._h)
            self._h = P()

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def params(self):
        p = self.np.empty(self.param_count(), self.np.float32)
        check(self.L.aphid_unet_get_params(self._h, p.ctypes.data), "unet_get_params")
        return p

    def set_params(self, p):
        p = self.np.ascontiguousarray(p, self.np.float32)
        assert p.size == self.param_count()
        check(self.L.aphid_unet_set_params(self._h, p.ctypes.data), "unet_set_params")

    def grads(self):
        g = self.np.empty(self.param_count(), self.np.float32)
        check(self.L.aphid_unet_get_grads(self._h, g.ctypes.data), "unet_get_grads")
        return g

    def forward(self, x, y, stream=None):
        """y [V][8] = net(x [V][3]) (float32 CUDA tensors)."""
        check(self.L.aphid_unet_forward(self._h, x.data_ptr(), y.data_ptr(), stream), "unet_forward")

    def train_step(self, x, target, weight=None, lr=1e-3, update=True, stream=None):
        loss = C.c_double()
        check(self.L.aphid_unet_train_step(self._h, x.data_ptr(), target.data_ptr(),
                                           weight.data_ptr() if weight is not None else None, lr,
                                           int(update), C.byref(loss), stream), "unet_train_step")
        return loss.value
