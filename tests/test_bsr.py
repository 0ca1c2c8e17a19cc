"""Block CSR (BSRMatrix, core/matrix.hpp:962-1060) on the CPU.

Three layers are checked here, each bit for bit:
  * the CPU restatement (oracle/raptor_oracle.c) against the reference's own
    compiled BSRMatrix (core/matrix.cpp, util/linalg/spmv.cpp; oracle/_ref),
    for the products mult / mult_append / residual / mult_T and to_CSR;
  * the per-row code the CUDA kernels run (raptor_b200/csrc/bsr.cuh), built
    for the host, against the restatement;
  * the host block COO -> block CSR conversion of the Python mirror against
    the reference's BCOOMatrix::to_BSR, and its sort / move_diag /
    remove_duplicates against the reference's (rows with distinct block
    columns; repeated ones are summed entry by entry, which the reference's
    block append_vals does not do).
The reference's own known-answer test for block matrices
(raptor/core/tests/test_block_matrix.cpp) is replayed on its fixture
(tests/golden/block_matrix.json): the block and the scalar forms of its
matrix give the same products and CSR entries.
"""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

import raptor_b200 as rb
from oracle import oracle as O
from tests.conftest import ROOT

CSRC = os.path.join(ROOT, "raptor_b200", "csrc")
FIXTURE = os.path.join(ROOT, "tests", "golden", "block_matrix.json")
OPS = {"mult": 0, "mult_append": 1, "residual": 2, "mult_T": 3}
SHAPES = [(1, 1), (2, 2), (3, 3), (2, 3), (4, 1), (1, 5)]


def random_bsr(nbr, nbc, br, bc, seed, per_row=4):
    """Block rows of 0..2*per_row blocks (some empty), repeated block columns
    inside a row, exact zeros and values below the 1e-16 drop tolerance."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(0, 2 * per_row + 1, nbr)
    counts[rng.random(nbr) < 0.1] = 0
    rowptr = np.zeros(nbr + 1, np.int32)
    rowptr[1:] = np.cumsum(counts)
    nnz = int(rowptr[-1])
    cols = rng.integers(0, nbc, nnz).astype(np.int32)
    blocks = rng.uniform(-1, 1, (nnz, br, bc))
    blocks[rng.random((nnz, br, bc)) < 0.15] = 0.0
    blocks[rng.random((nnz, br, bc)) < 0.05] = 3e-17
    return O.BSR(nbr, nbc, br, bc, rowptr, cols, blocks)


def vectors(A, seed):
    rng = np.random.default_rng(seed + 1000)
    n, m = A.shape
    return rng.uniform(-1, 1, m), rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)


def oracle_op(A, op, x, b, xt):
    if op == "mult":
        return O.bsr_spmv(A, x)
    if op == "mult_append":
        return O.bsr_append(A, x, b)
    if op == "residual":
        return O.bsr_residual(A, x, b)
    return O.bsr_spmv_T(A, xt)


# ------------------------------------------------------------ reference --
@pytest.fixture(scope="module")
def ref():
    L = O.ref_lib()
    if L is None:
        pytest.skip("the reference's sequential build is not available")
    return L


def ref_op(L, A, op, x, b, xt):
    rp, ci, v = A._args()
    n, m = A.shape
    out = np.zeros(m if op == "mult_T" else n)
    L.rs_bsr_apply(A.n_rows, A.n_cols, A.b_rows, A.b_cols, rp, ci, v, OPS[op],
                   np.ascontiguousarray(xt if op == "mult_T" else x),
                   np.ascontiguousarray(b if n else np.zeros(1)), out)
    return out


@pytest.mark.parametrize("br,bc", SHAPES)
@pytest.mark.parametrize("op", sorted(OPS))
def test_restatement_products_equal_reference(ref, br, bc, op):
    A = random_bsr(37, 29, br, bc, seed=br * 10 + bc)
    x, b, xt = vectors(A, br * 10 + bc)
    np.testing.assert_array_equal(oracle_op(A, op, x, b, xt), ref_op(ref, A, op, x, b, xt))


@pytest.mark.parametrize("br,bc", SHAPES)
def test_restatement_to_csr_equals_reference(ref, br, bc):
    A = random_bsr(41, 23, br, bc, seed=7 + br + 3 * bc)
    rp, ci, v = A._args()
    (n, m), rrp, rci, rcv = O.ref_take(ref.rs_bsr_to_csr(A.n_rows, A.n_cols, br, bc, rp, ci, v))
    B = O.bsr_to_csr(A)
    assert B.shape[:2] == (n, m) == A.shape
    orp, oci, ocv = B.arrays()
    np.testing.assert_array_equal(orp, rrp)
    np.testing.assert_array_equal(oci, rci)
    np.testing.assert_array_equal(ocv, rcv)


@pytest.mark.parametrize("br,bc", [(2, 2), (3, 2)])
def test_bcoo_to_bsr_equals_reference(ref, br, bc):
    rng = np.random.default_rng(5)
    nbr, nbc, nnz = 19, 17, 120
    rows = rng.integers(0, nbr, nnz).astype(np.int32)
    cols = rng.integers(0, nbc, nnz).astype(np.int32)
    vals = rng.uniform(-1, 1, (nnz, br, bc))
    rp = np.zeros(nbr + 1, np.int32)
    ci = np.zeros(nnz, np.int32)
    v = np.zeros(nnz * br * bc)
    ref.rs_bcoo_to_bsr(nbr, nbc, br, bc, nnz, rows, cols, np.ascontiguousarray(vals.reshape(-1)),
                       rp, ci, v)
    hrp, hci, hv = rb.bcoo_to_bsr_arrays(nbr, br, bc, rows, cols, vals)
    np.testing.assert_array_equal(hrp, rp)
    np.testing.assert_array_equal(hci, ci)
    np.testing.assert_array_equal(hv.reshape(-1), v)


# ----------------------------------------------- the kernels' row code --
@pytest.fixture(scope="module")
def host_rows(tmp_path_factory):
    out = tmp_path_factory.mktemp("bsr") / "libbsr_rows.so"
    subprocess.check_call(["g++", "-O2", "-std=c++14", "-ffp-contract=off", "-fPIC", "-shared",
                           "-I", CSRC, os.path.join(ROOT, "tests", "cxx", "bsr_rows.cpp"),
                           "-o", str(out)])
    L = C.CDLL(str(out))
    I = np.ctypeslib.ndpointer(np.int32, flags="C")
    D = np.ctypeslib.ndpointer(np.float64, flags="C")
    L.bsr_rows_apply.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, I, I, D, D, D, D]
    L.bsr_cols_T.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, I, I, D, D, D]
    L.bsr_csr_count.restype = C.c_int
    L.bsr_csr_count.argtypes = [C.c_int, C.c_int, C.c_int, I, D, I]
    L.bsr_csr_fill.argtypes = [C.c_int, C.c_int, C.c_int, I, I, D, I, I, D]
    return L


def host_op(L, A, op, x, b, xt):
    rp, ci, v = A._args()
    n, m = A.shape
    if op == "mult_T":
        out = np.zeros(max(m, 1))
        L.bsr_cols_T(A.n_rows, A.n_cols, A.b_rows, A.b_cols, rp, ci, v, np.ascontiguousarray(xt),
                     out)
        return out[:m]
    out = np.zeros(max(n, 1))
    L.bsr_rows_apply(OPS[op], A.n_rows, A.b_rows, A.b_cols, rp, ci, v, np.ascontiguousarray(x),
                     np.ascontiguousarray(b if n else np.zeros(1)), out)
    return out[:n]


@pytest.mark.parametrize("br,bc", SHAPES)
@pytest.mark.parametrize("op", sorted(OPS))
def test_kernel_rows_on_the_host_match_the_restatement(host_rows, br, bc, op):
    A = random_bsr(53, 31, br, bc, seed=100 + br * 10 + bc)
    x, b, xt = vectors(A, 3)
    np.testing.assert_array_equal(host_op(host_rows, A, op, x, b, xt), oracle_op(A, op, x, b, xt))


@pytest.mark.parametrize("br,bc", SHAPES)
def test_kernel_expansion_on_the_host_matches_the_restatement(host_rows, br, bc):
    A = random_bsr(47, 19, br, bc, seed=200 + br * 10 + bc)
    rp, ci, v = A._args()
    n = A.shape[0]
    out_rp = np.zeros(n + 1, np.int32)
    nnz = host_rows.bsr_csr_count(A.n_rows, br, bc, rp, v, out_rp)
    out_ci = np.zeros(max(nnz, 1), np.int32)
    out_v = np.zeros(max(nnz, 1))
    host_rows.bsr_csr_fill(A.n_rows, br, bc, rp, ci, v, out_rp, out_ci, out_v)
    orp, oci, ocv = O.bsr_to_csr(A).arrays()
    np.testing.assert_array_equal(out_rp, orp)
    np.testing.assert_array_equal(out_ci[:nnz], oci)
    np.testing.assert_array_equal(out_v[:nnz], ocv)


# -------------------------------------------- the reference's known answer --
def fixture_matrices():
    with open(FIXTURE) as f:
        fx = json.load(f)
    nbr, nbc = fx["block_num_rows"], fx["block_num_cols"]
    br, bc = fx["block_row_size"], fx["block_col_size"]
    rp, ci, blocks = rb.bcoo_to_bsr_arrays(nbr, br, bc, fx["block_rows"], fx["block_cols"],
                                           fx["vals"])
    A = O.BSR(nbr, nbc, br, bc, rp, ci, blocks)
    # COOMatrix::add_value(row, col, double) keeps |v| > 1e-16 (core/matrix.hpp:543-552)
    vals = np.asarray(fx["vals"])
    keep = np.abs(vals) > 1e-16
    dense = np.zeros((nbr * br, nbc * bc))
    np.add.at(dense, (np.asarray(fx["rows"])[keep], np.asarray(fx["cols"])[keep]), vals[keep])
    return fx, A, dense, int(keep.sum())


def test_fixture_block_and_scalar_forms_agree():
    """test_block_matrix.cpp: BSR and CSR products of ones agree (1e-10),
    and the BSR's CSR expansion has the scalar matrix's entries."""
    fx, A, dense, nnz = fixture_matrices()
    ones = np.ones(A.shape[1])
    np.testing.assert_allclose(O.bsr_spmv(A, ones), dense @ ones, rtol=0, atol=1e-10)
    np.testing.assert_allclose(O.bsr_spmv_T(A, ones), dense.T @ ones, rtol=0, atol=1e-10)
    B = O.bsr_to_csr(A)
    assert B.shape == (A.shape[0], A.shape[1], nnz)
    np.testing.assert_array_equal(B.to_scipy().toarray(), dense)
    assert A.rowptr.tolist() == [0, 2, 3, 5]   # the test's block_row_ptr


def test_fixture_matches_reference(ref):
    fx, A, dense, _ = fixture_matrices()
    x, b, xt = vectors(A, 11)
    for op in OPS:
        np.testing.assert_array_equal(oracle_op(A, op, x, b, xt), ref_op(ref, A, op, x, b, xt))


# ------------------------------------------------------------- boundary --
def test_bsr_entry_points_refuse_without_a_device():
    """No CPU fallback: creating a device block matrix fails loudly."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(rb.RaptorError) as e:
        rb.BSRMatrix.from_arrays(1, 1, 2, 2, [0, 1], [0], np.ones(4))
    assert e.value.code == -6


def test_bsr_arrays_are_checked_before_any_device_call():
    """Short arrays are refused by the mirror (RB_ERR_INVALID), so the C ABI
    never reads past them; no device is needed to see it."""
    for args in [(2, 2, 1, 1, [0, 1], [0], [1.0]),            # rowptr too short
                 (1, 2, 1, 1, [0, 2], [0], [1.0]),            # cols too short
                 (1, 2, 2, 2, [0, 1], [1], np.ones(3))]:      # values too short
        with pytest.raises(rb.RaptorError) as e:
            rb.BSRMatrix.from_arrays(*args)
        assert e.value.code == -1


def test_bsr_host_conversion_checks_its_input():
    with pytest.raises(rb.RaptorError):
        rb.bcoo_to_bsr_arrays(2, 1, 1, [0, 2], [0, 0], [1.0, 2.0])
    with pytest.raises(rb.RaptorError):
        rb.bcoo_to_bsr_arrays(2, 1, 1, [0, 1], [0], [1.0, 2.0])


# ------------------------------------------- sort, move_diag, remove_duplicates --
def random_distinct_bsr(nb, br, bc, seed):
    """Square block matrix whose block rows hold distinct block columns in
    random order (the diagonal block in about half of them), with all-zero
    blocks and blocks whose entries sum below the 1e-16 drop tolerance."""
    rng = np.random.default_rng(seed)
    rowptr, cols, blocks = [0], [], []
    for i in range(nb):
        k = int(rng.integers(0, 7))
        c = rng.choice(nb, size=min(k, nb), replace=False)
        if rng.random() < 0.5 and i not in c:
            c = np.append(c, i)
        rng.shuffle(c)
        cols.extend(c.tolist())
        rowptr.append(len(cols))
    blocks = rng.uniform(-1, 1, (len(cols), br, bc))
    pick = rng.random(len(cols))
    blocks[pick < 0.1] = 0.0
    blocks[(pick >= 0.1) & (pick < 0.15)] = 1e-18
    return O.BSR(nb, nb, br, bc, rowptr, cols, blocks)


@pytest.mark.parametrize("br,bc", [(1, 1), (2, 2), (3, 2)])
def test_sort_diag_first_equals_reference(ref, br, bc):
    A = random_distinct_bsr(60, br, bc, seed=br * 7 + bc)
    rp, ci, v = A._args()
    z = len(A.cols)
    out_rp = np.zeros(A.n_rows + 1, np.int32)
    out_ci = np.zeros(max(z, 1), np.int32)
    out_v = np.zeros(max(z * br * bc, 1))
    nnz = ref.rs_bsr_sort_diag_first(A.n_rows, A.n_cols, br, bc, rp, ci, v, out_rp, out_ci, out_v)
    hrp, hci, hv = rb.bsr_sort_diag_first(A.n_rows, br, bc, A.rowptr, A.cols, A.blocks)
    np.testing.assert_array_equal(hrp, out_rp)
    np.testing.assert_array_equal(hci, out_ci[:nnz])
    np.testing.assert_array_equal(hv.reshape(-1), out_v[:nnz * br * bc])


def test_sort_diag_first_sums_repeated_blocks():
    """Repeated block columns are summed entry by entry (where the reference
    adds the wrong entries): the matrix is unchanged, each row holds distinct
    columns with the diagonal block first, the rest in increasing order."""
    A = random_bsr(40, 40, 2, 3, seed=17, per_row=5)
    rp, ci, bl = rb.bsr_sort_diag_first(A.n_rows, 2, 3, A.rowptr, A.cols, A.blocks)
    B = O.BSR(40, 40, 2, 3, rp, ci, bl)
    np.testing.assert_allclose(O.bsr_to_csr(B).to_scipy().toarray(),
                               O.bsr_to_csr(A).to_scipy().toarray(), rtol=0, atol=1e-15)
    for i in range(40):
        row = ci[rp[i]:rp[i + 1]].tolist()
        rest = row[1:] if row and row[0] == i else row
        assert i not in rest and rest == sorted(set(rest))
    assert np.all(np.abs(bl).reshape(len(ci), -1).sum(axis=1) >= 1e-16)


def test_fixture_sort_diag_first_equals_reference(ref):
    """test_block_matrix.cpp sorts, moves the diagonal and removes duplicates
    of its block matrix before comparing it with the scalar form."""
    _, A, dense, _ = fixture_matrices()
    rp, ci, v = A._args()
    z = len(A.cols)
    out_rp = np.zeros(A.n_rows + 1, np.int32)
    out_ci = np.zeros(z, np.int32)
    out_v = np.zeros(z * A.b_rows * A.b_cols)
    nnz = ref.rs_bsr_sort_diag_first(A.n_rows, A.n_cols, A.b_rows, A.b_cols, rp, ci, v, out_rp,
                                     out_ci, out_v)
    hrp, hci, hv = rb.bsr_sort_diag_first(A.n_rows, A.b_rows, A.b_cols, A.rowptr, A.cols,
                                          A.blocks)
    np.testing.assert_array_equal(hrp, out_rp)
    np.testing.assert_array_equal(hci, out_ci[:nnz])
    np.testing.assert_array_equal(hv.reshape(-1), out_v[:nnz * A.b_rows * A.b_cols])
    B = O.BSR(A.n_rows, A.n_cols, A.b_rows, A.b_cols, hrp, hci, hv)
    np.testing.assert_array_equal(O.bsr_to_csr(B).to_scipy().toarray(), dense)


def test_bench_block_pattern_is_in_bounds():
    """bench.py's block CSR workload: 7 distinct in-range block columns a
    block row, the diagonal block first, and the CLI default cases parse."""
    import sys

    import bench
    rowptr, cols = bench.block_stencil_pattern(6)
    nb = 6 ** 3
    assert rowptr[0] == 0 and rowptr[-1] == len(cols) == 7 * nb
    assert cols.min() >= 0 and cols.max() < nb
    per_row = cols.reshape(nb, 7)
    assert np.array_equal(per_row[:, 0], np.arange(nb))
    assert all(len(set(r)) == 7 for r in per_row.tolist())
    argv = sys.argv
    try:
        sys.argv = ["bench.py"]
        cases = bench.parse().bsr_cases
    finally:
        sys.argv = argv
    assert [tuple(int(v) for v in c.split("x")) for c in cases.split(",")] == [
        (96, 3), (112, 2), (64, 4)]
