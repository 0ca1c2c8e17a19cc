"""Block CSR on the GPU through the C ABI (rb_bsr_*): the products, the
transposed product (twice: the second call reuses the transposed block
pattern kept on the handle) and the expansion to CSR equal the CPU
restatement bit for bit; the restatement equals the reference's own
BSRMatrix bit for bit (tests/test_bsr.py).  Also the reference's
known-answer matrix (test_block_matrix.cpp), empty block rows and a
matrix without blocks, and the errors a caller gets for mismatched sizes."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import ROOT
from tests.test_bsr import SHAPES, oracle_op, random_bsr, vectors

pytestmark = pytest.mark.gpu

rb = pytest.importorskip("raptor_b200")


@pytest.fixture(scope="module", autouse=True)
def _device():
    rb.init(0)


def to_rb(A):
    return rb.BSRMatrix.from_arrays(A.n_rows, A.n_cols, A.b_rows, A.b_cols, A.rowptr, A.cols,
                                    A.blocks)


def gpu_op(M, A, op, x, b, xt):
    n, m = A.shape
    if op == "mult_T":
        out = rb.ParVector(m)
        M.mult_T(rb.ParVector(n, values=xt), out)
        return out.numpy()
    xv = rb.ParVector(m, values=x)
    if op == "mult":
        out = rb.ParVector(n)
        M.mult(xv, out)
    elif op == "mult_append":
        out = rb.ParVector(n, values=b)
        M.mult_append(xv, out)
    else:
        out = rb.ParVector(n)
        M.residual(xv, rb.ParVector(n, values=b), out)
    return out.numpy()


@pytest.mark.parametrize("br,bc", SHAPES)
def test_products_equal_the_restatement(br, bc):
    A = random_bsr(301, 257, br, bc, seed=400 + br * 10 + bc, per_row=6)
    M = to_rb(A)
    assert M.info() == (A.n_rows, A.n_cols, br, bc, len(A.cols))
    rp, ci, blocks = M.arrays()
    np.testing.assert_array_equal(rp, A.rowptr)
    np.testing.assert_array_equal(ci, A.cols)
    np.testing.assert_array_equal(blocks, A.blocks)
    x, b, xt = vectors(A, 9)
    for op in ("mult", "mult_append", "residual", "mult_T", "mult_T"):
        np.testing.assert_array_equal(gpu_op(M, A, op, x, b, xt), oracle_op(A, op, x, b, xt),
                                      err_msg=op)


@pytest.mark.parametrize("br,bc", SHAPES)
def test_to_csr_equals_the_restatement(br, bc):
    A = random_bsr(211, 173, br, bc, seed=500 + br * 10 + bc, per_row=5)
    B = to_rb(A).to_CSR()
    assert B.info()[:2] == A.shape
    grp, gci, gcv = B.arrays()
    orp, oci, ocv = O.bsr_to_csr(A).arrays()
    np.testing.assert_array_equal(grp, orp)
    np.testing.assert_array_equal(gci, oci)
    np.testing.assert_array_equal(gcv, ocv)


def test_reference_known_answer_matrix():
    """test_block_matrix.cpp's matrix, built from its blocks on the host and
    multiplied on the GPU: the scalar matrix's products and entries."""
    with open(os.path.join(ROOT, "tests", "golden", "block_matrix.json")) as f:
        fx = json.load(f)
    nbr, nbc = fx["block_num_rows"], fx["block_num_cols"]
    br, bc = fx["block_row_size"], fx["block_col_size"]
    M = rb.BSRMatrix.from_blocks(nbr, nbc, br, bc, fx["block_rows"], fx["block_cols"], fx["vals"])
    vals = np.asarray(fx["vals"])
    keep = np.abs(vals) > 1e-16
    dense = np.zeros((nbr * br, nbc * bc))
    np.add.at(dense, (np.asarray(fx["rows"])[keep], np.asarray(fx["cols"])[keep]), vals[keep])
    ones = rb.ParVector(nbc * bc)
    ones.set_const_value(1.0)
    out = rb.ParVector(nbr * br)
    M.mult(ones, out)
    np.testing.assert_allclose(out.numpy(), dense.sum(axis=1), rtol=0, atol=1e-10)
    M.mult_T(ones, out)
    np.testing.assert_allclose(out.numpy(), dense.sum(axis=0), rtol=0, atol=1e-10)
    C = M.to_CSR()
    assert C.info()[2] == int(keep.sum())
    np.testing.assert_array_equal(C.to_scipy().toarray(), dense)


def test_matrix_without_blocks():
    A = O.BSR(5, 4, 2, 3, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros((0, 2, 3)))
    M = to_rb(A)
    x, b, xt = vectors(A, 1)
    for op in ("mult", "mult_append", "residual", "mult_T"):
        np.testing.assert_array_equal(gpu_op(M, A, op, x, b, xt), oracle_op(A, op, x, b, xt),
                                      err_msg=op)
    assert M.to_CSR().info() == (10, 12, 0)


def test_errors_are_status_codes():
    A = random_bsr(12, 9, 2, 3, seed=3)
    M = to_rb(A)
    with pytest.raises(rb.RaptorError):
        M.mult(rb.ParVector(A.shape[0]), rb.ParVector(A.shape[0]))   # x has the wrong size
    x = rb.ParVector(A.shape[1])
    with pytest.raises(rb.RaptorError):
        M.mult_T(x, x)
    with pytest.raises(rb.RaptorError):
        rb.BSRMatrix.from_arrays(2, 2, 2, 2, [0, 1, 1], [2], np.ones(4))   # column out of range
    with pytest.raises(rb.RaptorError):
        rb.BSRMatrix.from_arrays(2, 2, 0, 2, [0, 0, 0], [], np.ones(0))    # zero block rows
