"""Edge cases through the C ABI: empty and one-row systems, ragged rows (one
very long row, empty rows), a hierarchy that is only its coarse level, and
the errors a caller gets for mismatched or missing arguments (negative status
codes, never a crash or a silent CPU path)."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O
from tests.test_gpu_parity import assert_csr_equal, oc_tuple, rb_tuple, to_rb

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")


@pytest.fixture(scope="module", autouse=True)
def _device():
    rb.init(0)


def ragged(n, seed, long_row=True, empty_rows=True):
    """SPD-ish random matrix with uneven rows: a few empty rows, one row
    (and column) with thousands of entries, diagonal dominant elsewhere."""
    rng = np.random.default_rng(seed)
    M = sp.random(n, n, density=4.0 / n, random_state=seed, format="lil")
    if long_row:
        cols = rng.choice(n, size=min(n - 1, 3000), replace=False)
        M[n // 2, cols] = rng.uniform(-1, 0, len(cols))
    M = sp.csr_matrix(M)
    M = -abs(M + M.T)
    M.setdiag(0)
    M.eliminate_zeros()
    d = np.asarray(abs(M).sum(axis=1)).ravel() + 1.0
    M = M + sp.diags(d)
    M = sp.csr_matrix(M)
    if empty_rows:
        for r in (3, 7):
            M.data[M.indptr[r]:M.indptr[r + 1]] = 0.0
        M.eliminate_zeros()
    M.sort_indices()
    return M


def oc_from_scipy(M):
    return O.CSR.from_arrays(M.shape[0], M.shape[1], M.indptr.astype(np.int32),
                             M.indices.astype(np.int32), M.data.astype(np.float64))


def test_spmv_family_on_ragged_rows_is_exact():
    M = ragged(6000, 1)
    A = rb.ParCSRMatrix.from_scipy(M)
    Ao = oc_from_scipy(M)
    n = M.shape[0]
    x = np.random.default_rng(2).uniform(-1, 1, n)
    b = np.random.default_rng(3).uniform(-1, 1, n)
    xv, bv, yv = rb.ParVector(n, values=x), rb.ParVector(n, values=b), rb.ParVector(n)
    A.mult(xv, yv)
    np.testing.assert_allclose(yv.numpy(), O.spmv(Ao, x), rtol=1e-13, atol=1e-13)
    A.residual(xv, bv, yv)
    np.testing.assert_allclose(yv.numpy(), O.residual(Ao, x, b), rtol=1e-13, atol=1e-13)
    A.mult_T(xv, yv)
    np.testing.assert_allclose(yv.numpy(), O.spmv_T(Ao, x), rtol=1e-13, atol=1e-13)


def test_spgemm_with_a_long_row_uses_the_global_bins_exactly():
    # the 3000-entry row and column produce product rows too long for the
    # shared-memory hash tables
    M = ragged(5000, 4, empty_rows=False)
    A = rb.ParCSRMatrix.from_scipy(M)
    Ao = oc_from_scipy(M)
    got = A.mult_matrix(A)
    ref = O.spgemm(Ao, Ao)
    assert_csr_equal(rb_tuple(got), oc_tuple(ref), exact_order=False)


def test_one_row_and_coarse_only_hierarchies():
    # 1 x 1: the hierarchy is the dense solve, PCG converges at once
    A = rb.ParCSRMatrix.from_arrays(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32),
                                    np.array([4.0]))
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    ml.setup(A)
    assert ml.num_levels == 1
    x = rb.ParVector(1)
    res = []
    rb.PCG(A, ml, x, rb.ParVector(1, values=np.array([2.0])), res, tol=1e-12,
           mode=rb.PCG_TRUE_RESIDUAL)
    assert abs(x.numpy()[0] - 0.5) < 1e-15
    # max_coarse above n: one level, the solve is the direct solve
    Ao = O.stencil_grid(O.laplace_stencil_27pt(), [3, 3, 3])
    A = to_rb(Ao)
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    ml.max_coarse = 100
    ml.setup(A)
    assert ml.num_levels == 1
    x = rb.ParVector(27)
    bh = np.arange(27.0)
    it = ml.solve(x, rb.ParVector(27, values=bh))
    assert it == 1
    np.testing.assert_allclose(O.spmv(Ao, x.numpy()), bh, rtol=1e-12, atol=1e-12)


def test_empty_system():
    A = rb.ParCSRMatrix.from_arrays(0, 0, np.array([0], np.int32), np.zeros(0, np.int32),
                                    np.zeros(0))
    x, b = rb.ParVector(0), rb.ParVector(0)
    A.mult(x, b)
    assert b.norm(2) == 0.0


def test_errors_are_status_codes():
    L = rb.lib()
    Ao = O.stencil_grid(O.laplace_stencil_27pt(), [4, 4, 4])
    A = to_rb(Ao)
    x, y = rb.ParVector(64), rb.ParVector(63)
    assert L.rb_spmv(A.h, x.h, y.h) == -1                      # size mismatch
    assert "size" in rb.last_error() or "match" in rb.last_error()
    assert L.rb_spmv(None, x.h, x.h) == -1                      # NULL handle
    R = rb.ParCSRMatrix.from_arrays(2, 3, np.array([0, 1, 2], np.int32),
                                    np.array([0, 2], np.int32), np.array([1.0, 1.0]))
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    with pytest.raises(rb.RaptorError):                         # AMG needs a square matrix
        ml.setup(R)
    opts = rb.AmgOpts()
    L.rb_amg_default_opts(C.byref(opts))
    opts.solver = 7
    h = C.c_void_p()
    assert L.rb_amg_setup(A.h, C.byref(opts), None, C.byref(h)) == -1
    ml = rb.ParRugeStubenSolver(0.25, rb.PMIS, rb.Extended, rb.Classical, rb.L1Jacobi)
    ml.setup(A)
    bad = C.c_double()
    assert L.rb_amg_time_operator(ml.h, 0, 9, 3, C.byref(bad)) == -1   # unknown operator
    assert L.rb_amg_level_info(ml.h, 99, None, None, None) == -1       # level out of range


def test_mult_T_reuses_its_transpose_and_follows_value_changes():
    """rb_spmv_T keeps A^T's pattern on the handle after the first call and
    gathers A's current values through it; reordering the rows
    (sort_diag_first) drops the kept pattern."""
    Ao = O.stencil_grid(O.diffusion_stencil_2d(0.001, np.pi / 8), [37, 23])
    n, m, _ = Ao.shape
    rp, ci, cv = Ao.arrays()
    A = rb.ParCSRMatrix.from_arrays(n, m, rp, ci, cv)
    xh = np.random.default_rng(4).uniform(-1, 1, n)
    x = rb.ParVector(n, values=xh)
    y = rb.ParVector(m)
    for _ in range(2):
        A.mult_T(x, y)
        np.testing.assert_allclose(y.numpy(), O.spmv_T(Ao, xh), rtol=1e-13, atol=1e-14)
    allocs = C.c_int64()
    rb.check(rb.lib().rb_device_alloc_count(C.byref(allocs)))
    A.mult_T(x, y)
    after = C.c_int64()
    rb.check(rb.lib().rb_device_alloc_count(C.byref(after)))
    assert after.value == allocs.value
    # new values through the borrowed device pointers
    torch = pytest.importorskip("torch")
    p_rp, p_ci, p_cv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    rb.check(rb.lib().rb_csr_device_arrays(A.h, C.byref(p_rp), C.byref(p_ci), C.byref(p_cv)))
    cv2 = cv * 1.5 + 0.25

    class _Vals:  # the library's value array as a torch tensor (no copy)
        __cuda_array_interface__ = {"shape": (len(cv2),), "typestr": "<f8",
                                    "data": (p_cv.value, False), "version": 3}

    rb.check(rb.lib().rb_synchronize())
    torch.as_tensor(_Vals(), device="cuda").copy_(torch.from_numpy(cv2))
    torch.cuda.synchronize()
    A.mult_T(x, y)
    Ao2 = O.CSR.from_arrays(n, m, rp, ci, cv2)
    np.testing.assert_allclose(y.numpy(), O.spmv_T(Ao2, xh), rtol=1e-13, atol=1e-14)
    A.sort_diag_first()
    A.mult_T(x, y)
    np.testing.assert_allclose(y.numpy(), O.spmv_T(Ao2, xh), rtol=1e-13, atol=1e-14)
