"""Failure paths of the Krylov solvers, made on the host (no GPU fault).

The reference's PCG prints "Indefinite matrix detected in CG! Aborting..."
and calls exit(-1) when p.Ap < 0 (raptor/krylov/par_cg.cpp:195-202); here
every solver returns RB_ERR_BREAKDOWN instead (the Python mirror raises
Breakdown), with the history up to that point.  A right-hand side holding a
NaN breaks down the same way, and an iteration limit reached before the
tolerance returns RB_ERR_NOT_CONVERGED with the partial history.  The
failures come from the inputs only: a negative definite operator, a NaN in
b, a small max_iter.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")


@pytest.fixture(scope="module", autouse=True)
def _device():
    rb.init(0)


def poisson5(m, sign=1.0):
    """sign * (5-point Laplacian) on an m x m grid (SPD for sign = 1,
    negative definite for sign = -1)."""
    st = [0.0, -1.0, 0.0, -1.0, 4.0, -1.0, 0.0, -1.0, 0.0]
    A = rb.par_stencil_grid(st, [m, m])
    n = A.global_num_rows
    rp, ci, cv = A.arrays()
    return rb.ParCSRMatrix.from_arrays(n, n, rp, ci, sign * cv)


def hierarchy(A, prec=rb.FP64):
    """RS AMG; a negative definite operator has no strong connections in the
    classical sense, so its hierarchy is kept to the direct coarse solve
    (max_coarse above its size): the preconditioner is then A^-1 itself."""
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    ml.precision = prec
    ml.max_coarse = 2000
    ml.setup(A)
    return ml


@pytest.mark.parametrize("mode", [rb.PCG_REFERENCE, rb.PCG_TRUE_RESIDUAL],
                         ids=["reference_mode", "true_residual_mode"])
@pytest.mark.parametrize("prec", [rb.FP64, rb.FP32], ids=["fp64", "fp32"])
def test_pcg_negative_definite_breaks_down(mode, prec):
    A = poisson5(40, -1.0)
    ml = hierarchy(A, prec)
    n = A.global_num_rows
    b = rb.ParVector(n, values=np.random.default_rng(1).uniform(-1, 1, n))
    x = rb.ParVector(n)
    res = []
    with pytest.raises(rb.Breakdown):
        rb.PCG(A, ml, x, b, res, tol=1e-8, max_iter=50, mode=mode)
    assert len(res) >= 1


@pytest.mark.parametrize("mode", [rb.PCG_REFERENCE, rb.PCG_TRUE_RESIDUAL],
                         ids=["reference_mode", "true_residual_mode"])
def test_pcg_nan_right_hand_side_breaks_down(mode):
    A = poisson5(64)
    ml = hierarchy(A)
    n = A.global_num_rows
    bh = np.random.default_rng(2).uniform(-1, 1, n)
    bh[n // 3] = math.nan
    b = rb.ParVector(n, values=bh)
    x = rb.ParVector(n)
    with pytest.raises(rb.Breakdown):
        rb.PCG(A, ml, x, b, [], tol=1e-8, max_iter=50, mode=mode)


@pytest.mark.parametrize("mode,entries", [(rb.PCG_REFERENCE, 3), (rb.PCG_TRUE_RESIDUAL, 3)],
                         ids=["reference_mode", "true_residual_mode"])
def test_pcg_iteration_limit_returns_not_converged(mode, entries):
    A = poisson5(64)
    ml = hierarchy(A)
    n = A.global_num_rows
    b = rb.ParVector(n, values=np.random.default_rng(3).uniform(-1, 1, n))
    x = rb.ParVector(n)
    res = []
    rc = rb.PCG(A, ml, x, b, res, tol=1e-14, max_iter=2, mode=mode)
    assert rc == -5
    assert len(res) == entries
    assert all(np.isfinite(res))
    # the iterate is the one after two iterations, not a reset or a NaN
    assert np.all(np.isfinite(x.numpy())) and np.linalg.norm(x.numpy()) > 0


def test_block_pcg_negative_definite_breaks_down():
    A = poisson5(40, -1.0)
    ml = hierarchy(A, rb.FP32)
    n = A.global_num_rows
    k = 4
    B = rb.ParVector(n * k, values=np.random.default_rng(4).uniform(-1, 1, n * k))
    X = rb.ParVector(n * k)
    with pytest.raises(rb.Breakdown):
        rb.PCG_block(A, ml, X, B, k, tol=1e-8, max_iter=50)


def test_block_pcg_iteration_limit_returns_not_converged():
    A = poisson5(64)
    ml = hierarchy(A, rb.FP32)
    n = A.global_num_rows
    k = 2
    B = rb.ParVector(n * k, values=np.random.default_rng(5).uniform(-1, 1, n * k))
    X = rb.ParVector(n * k)
    rc, iters, relres = rb.PCG_block(A, ml, X, B, k, tol=1e-14, max_iter=2)
    assert rc == -5
    assert list(iters) == [2, 2] and np.all(relres > 1e-14)


def test_batch_pcg_with_a_negative_definite_member_breaks_down():
    mats = [poisson5(48), poisson5(40, -1.0), poisson5(33)]
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    ml.precision = rb.FP32
    ml.max_coarse = 2000
    Bt = rb.Batch(mats, ml)
    N = Bt.total_rows
    b = rb.ParVector(N, values=np.random.default_rng(6).uniform(-1, 1, N))
    x = rb.ParVector(N)
    with pytest.raises(rb.Breakdown):
        Bt.pcg(x, b, tol=1e-8, max_iter=50)


def test_batch_pcg_iteration_limit_returns_not_converged():
    mats = [poisson5(48), poisson5(33)]
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    ml.precision = rb.FP32
    Bt = rb.Batch(mats, ml)
    N = Bt.total_rows
    b = rb.ParVector(N, values=np.random.default_rng(7).uniform(-1, 1, N))
    x = rb.ParVector(N)
    rc, iters, relres = Bt.pcg(x, b, tol=1e-14, max_iter=2)
    assert rc == -5
    assert list(iters) == [2, 2] and np.all(relres > 1e-14)
