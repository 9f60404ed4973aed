"""aphid_git_b200 -- B200-native (sm_100a) APhiD frequency-domain solve.

The matrix-free Lorenz-gauged A-Phi operator on the staggered Yee grid and
the Jacobi-preconditioned complex-symmetric QMR that inverts it, as
hand-written CUDA kernels behind the C ABI of include/aphid_gpu.h.

    from aphid_git_b200 import Solver, model
    s = Solver()
    s.set_nodes(xn, yn, zn)
    k2 = s.gen_k2(model.sigma_hat("R", w, sig_re), w)
    x, info, hist = s.qmr(k2, s.gen_diag(k2), b, 1e-8, 2000)
"""
from . import model
from .abi import AphidError, Info, Solver, load, library_path

__all__ = ["AphidError", "Info", "Solver", "load", "library_path", "model"]
