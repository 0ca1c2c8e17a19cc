"""torch.autograd harness for the differentiation form.

``DiffusionSolve.apply(k, b, nx, ny)`` returns x = A(k)^-1 b, where A(k) is
the finite-volume operator rb_fv_assemble builds from the cell
conductivities k (harmonic-mean faces, Dirichlet walls), solved by
AMG-preconditioned CG (FP32 V-cycle, FP64 outer iteration, true relative
residual below ``tol``).  Its backward pass returns

    dL/db = lambda,  A^T lambda = dL/dx           (rb_adjoint_solve)
    dL/dk = assembly backward of  dL/dA_ij = -lambda_i x_j   (rb_sddmm, rb_fv_backward)

all through the C ABI on the tensors' device memory.  The hierarchy built in
the forward pass is reused by the adjoint solve.

``grf(nx, ny, corr_len, seed)`` draws the Gaussian random field of the
differentiation workload (spectral method, host numpy; see its docstring).
"""
import ctypes as C
import math

import numpy as np

from . import (FP32, PCG_TRUE_RESIDUAL, Extended, L1Jacobi, ParCSRMatrix, ParRugeStubenSolver,
               ParVector, PMIS, Classical, PCG, check, lib)


def grf(nx, ny, corr_len=32.0, seed=0):
    """A stationary Gaussian random field on an nx x ny cell grid with zero
    mean, unit variance and squared-exponential covariance
    exp(-r^2 / (2 corr_len^2)) (r in cells).

    Spectral method: white noise on a periodic grid padded by 4 corr_len in
    each direction (so the periodic wrap-around does not correlate opposite
    edges), multiplied in Fourier space by the square root of the
    covariance's discrete spectrum, transformed back and cropped.  The
    scaling divides by the field's exact (pre-crop) standard deviation, so the
    variance is one in expectation."""
    pad = int(math.ceil(4 * corr_len))
    mx, my = nx + pad, ny + pad
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((my, mx))
    # discrete covariance on the periodic grid, then its spectrum
    dx = np.minimum(np.arange(mx), mx - np.arange(mx)).astype(np.float64)
    dy = np.minimum(np.arange(my), my - np.arange(my)).astype(np.float64)
    cov = np.exp(-(dy[:, None] ** 2 + dx[None, :] ** 2) / (2.0 * corr_len ** 2))
    spec = np.maximum(np.fft.fft2(cov).real, 0.0)
    g = np.fft.ifft2(np.fft.fft2(w) * np.sqrt(spec)).real
    # variance of a sample: sum(spec) / (mx my) = cov(0) = 1 up to clipping
    g /= math.sqrt(spec.sum() / (mx * my))
    return np.ascontiguousarray(g[:ny, :nx].reshape(-1))


def _ptr(t):
    return C.c_void_p(t.data_ptr())


_dev_copy = None


def _copy_fns():
    """rb_vec_upload / rb_vec_download bound with pointer arguments (the
    shared binding takes numpy arrays); both accept device memory."""
    global _dev_copy
    if _dev_copy is None:
        L = C.CDLL(lib()._name)
        up, down = L.rb_vec_upload, L.rb_vec_download
        for f in (up, down):
            f.restype = C.c_int
            f.argtypes = [C.c_void_p, C.c_void_p]
        _dev_copy = (up, down)
    return _dev_copy


def _rb_sync():
    check(lib().rb_synchronize())


class DiffusionSolve:
    """A torch.autograd.Function (created lazily so importing this module
    does not import torch)."""

    _fn = None

    @classmethod
    def apply(cls, k, b, nx, ny, tol=1e-10, max_iter=500, precision=FP32):
        if cls._fn is None:
            cls._fn = _make_function()
        return cls._fn.apply(k, b, nx, ny, tol, max_iter, precision)


def _make_function():
    import torch

    class _Solve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, k, b, nx, ny, tol, max_iter, precision):
            assert k.dtype == torch.float64 and b.dtype == torch.float64 and k.is_cuda
            n = nx * ny
            k = k.contiguous()
            torch.cuda.current_stream().synchronize()
            h = C.c_void_p()
            check(lib().rb_fv_assemble(int(nx), int(ny), _ptr(k), C.byref(h)))
            A = ParCSRMatrix(h)
            ml = ParRugeStubenSolver(0.25, PMIS, Extended, Classical, L1Jacobi)
            ml.precision = precision
            ml.setup(A)
            bv = ParVector(n)
            bc = b.contiguous()
            check(_copy_fns()[0](bv.h, _ptr(bc)))
            xv = ParVector(n)
            res = []
            rc = PCG(A, ml, xv, bv, res, tol=tol, max_iter=max_iter, mode=PCG_TRUE_RESIDUAL)
            if rc != 0:
                raise RuntimeError("forward solve did not converge (%d)" % rc)
            x = torch.empty(n, dtype=torch.float64, device=k.device)
            check(_copy_fns()[1](xv.h, _ptr(x)))
            ctx.save_for_backward(k, x)
            ctx.A, ctx.ml, ctx.nx, ctx.ny = A, ml, nx, ny
            ctx.tol, ctx.max_iter = tol, max_iter
            ctx.forward_iters = len(res) - 1
            return x

        @staticmethod
        def backward(ctx, gx):
            k, x = ctx.saved_tensors
            A, ml, nx, ny = ctx.A, ctx.ml, ctx.nx, ctx.ny
            n = nx * ny
            torch.cuda.current_stream().synchronize()
            gv = ParVector(n)
            gxc = gx.contiguous().to(torch.float64)
            check(_copy_fns()[0](gv.h, _ptr(gxc)))
            lv = ParVector(n)
            it, rr = C.c_int(), C.c_double()
            rc = lib().rb_adjoint_solve(A.h, ml.h, lv.h, gv.h, float(ctx.tol), int(ctx.max_iter),
                                        C.byref(it), C.byref(rr))
            if rc != 0:
                raise RuntimeError("adjoint solve did not converge (%d)" % rc)
            lam = torch.empty(n, dtype=torch.float64, device=k.device)
            check(_copy_fns()[1](lv.h, _ptr(lam)))
            gA = torch.empty(A.local_nnz, dtype=torch.float64, device=k.device)
            check(lib().rb_sddmm(A.h, _ptr(lam), _ptr(x), -1.0, _ptr(gA)))
            gk = torch.empty(n, dtype=torch.float64, device=k.device)
            check(lib().rb_fv_backward(int(nx), int(ny), _ptr(k), A.h, _ptr(gA), _ptr(gk)))
            _rb_sync()
            return gk, lam, None, None, None, None, None

    return _Solve
