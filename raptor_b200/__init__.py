"""raptor_b200 -- RAPtor's algebraic-multigrid solve path on one B200.

A Python mirror of the reference's C++ API (13manan/raptor, world size 1)
over the C ABI of libraptor_b200.so.  Names, argument meaning and error
behaviour follow the reference:

    A = par_stencil_grid(laplace_stencil_27pt(), [n, n, n])   # gallery/par_stencil.hpp
    x = ParVector(A.global_num_rows); b = ParVector(A.global_num_rows)
    x.set_const_value(1.0); A.mult(x, b); x.set_const_value(0.0)
    ml = ParRugeStubenSolver(0.25, PMIS, Extended, Classical, L1Jacobi)
    ml.setup(A)
    res = []
    PCG(A, ml, x, b, res, tol=1e-8)                             # krylov/par_cg.hpp

Every computation runs in the CUDA library; importing works without a GPU,
but any compute call then raises RaptorError(RB_ERR_NO_DEVICE).
"""
import ctypes as C

import numpy as np

from ._capi import (AmgOpts, Breakdown, NotConverged, RaptorError, check, lib,  # noqa: F401
                    last_error)

# enums (core/types.hpp:158-164) --------------------------------------------
Classical, Symmetric = 0, 1                 # strength_t
RS, CLJP, Falgout, PMIS, HMIS = 0, 1, 2, 3, 4   # coarsen_t
Direct, ModClassical, Extended = 0, 1, 2    # interp_t
Jacobi, SOR, SSOR, L1Jacobi = 0, 1, 2, 3    # relax_t (+ L1-Jacobi)
MIS = 0                                     # agg_t
JacobiProlongation = 0                      # prolong_t
FP64, FP32 = 0, 1                           # cycle precision
PCG_REFERENCE, PCG_TRUE_RESIDUAL = 0, 1


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class ParVector:
    """Device FP64 vector (core/par_vector.hpp:44-176)."""

    def __init__(self, global_n, local_n=None, first_local=0, values=None):
        self.global_n = int(global_n)
        self.local_n = self.global_n if local_n is None else int(local_n)
        h = C.c_void_p()
        check(lib().rb_vec_create(self.local_n, C.byref(h)))
        self.h = h
        if values is not None:
            self.set_values(values)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().rb_vec_destroy(self.h)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self.h = None

    def __len__(self):
        return self.local_n

    def set_values(self, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        if v.shape != (self.local_n,):
            raise RaptorError(-1, "vector size mismatch")
        check(lib().rb_vec_upload(self.h, v))
        return self

    def numpy(self):
        out = np.empty(self.local_n, dtype=np.float64)
        check(lib().rb_vec_download(self.h, out))
        return out

    def set_const_value(self, v):
        check(lib().rb_vec_set(self.h, float(v)))

    def set_rand_values(self, seed=0):
        self.set_values(np.random.default_rng(seed).random(self.local_n))

    def copy(self, y):
        check(lib().rb_vec_copy(self.h, y.h))

    def axpy(self, x, alpha):
        check(lib().rb_vec_axpy(self.h, x.h, float(alpha)))

    def scale(self, alpha):
        check(lib().rb_vec_scale(self.h, float(alpha)))

    def inner_product(self, x):
        out = C.c_double()
        check(lib().rb_vec_dot(self.h, x.h, C.byref(out)))
        return out.value

    def norm(self, p=2):
        if p != 2:
            return float(np.linalg.norm(self.numpy(), p))
        out = C.c_double()
        check(lib().rb_vec_norm2(self.h, C.byref(out)))
        return out.value

    def device_ptr(self):
        p = C.c_void_p()
        check(lib().rb_vec_device_ptr(self.h, C.byref(p)))
        return p.value

    def torch_view(self):
        """The vector's device memory as a torch CUDA tensor (no copy; the
        vector must outlive the tensor).  Used to receive halo values
        straight into a vector."""
        import torch

        class _Cai:
            pass

        o = _Cai()
        o.__cuda_array_interface__ = {"shape": (self.local_n,), "typestr": "<f8",
                                      "data": (self.device_ptr(), False), "version": 3}
        return torch.as_tensor(o, device="cuda")

    def scatter_add(self, idx_dev, vals_dev, n):
        """self[idx[k]] += vals[k] for k < n (device pointers; distinct
        indices), on the library stream."""
        check(lib().rb_vec_scatter_add(self.h, C.c_void_p(idx_dev), C.c_void_p(vals_dev), int(n)))

    def gather(self, idx_dev, n, out_dev):
        """out[k] = self[idx[k]] for k < n (device pointers), on the library
        stream: a halo exchange's send-buffer packing."""
        check(lib().rb_vec_gather(self.h, C.c_void_p(idx_dev), int(n), C.c_void_p(out_dev)))


class ParCSRMatrix:
    """Device CSR matrix, FP64 values, int32 indices (core/par_matrix.hpp:481-611)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def from_arrays(cls, n_rows, n_cols, rowptr, cols, vals):
        rp = np.ascontiguousarray(rowptr, dtype=np.int32)
        ci = np.ascontiguousarray(cols, dtype=np.int32)
        cv = np.ascontiguousarray(vals, dtype=np.float64)
        if ci.size == 0:
            ci = np.zeros(1, np.int32)
            cv = np.zeros(1, np.float64)
        h = C.c_void_p()
        check(lib().rb_csr_create(int(n_rows), int(n_cols), int(rp[-1]), _ptr(rp), _ptr(ci),
                                  _ptr(cv), 0, C.byref(h)))
        return cls(h)

    @classmethod
    def from_scipy(cls, M):
        M = M.tocsr()
        return cls.from_arrays(M.shape[0], M.shape[1], M.indptr, M.indices, M.data)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().rb_csr_destroy(self.h)
            except Exception:  # noqa: BLE001
                pass
            self.h = None

    def info(self):
        r, c, z = C.c_int(), C.c_int(), C.c_int64()
        check(lib().rb_csr_info(self.h, C.byref(r), C.byref(c), C.byref(z)))
        return r.value, c.value, z.value

    @property
    def global_num_rows(self):
        return self.info()[0]

    @property
    def global_num_cols(self):
        return self.info()[1]

    @property
    def local_nnz(self):
        return self.info()[2]

    def arrays(self):
        n, m, z = self.info()
        rp = np.zeros(n + 1, np.int32)
        ci = np.zeros(max(z, 1), np.int32)
        cv = np.zeros(max(z, 1), np.float64)
        check(lib().rb_csr_download(self.h, _ptr(rp), _ptr(ci), _ptr(cv)))
        return rp, ci[:z], cv[:z]

    def to_scipy(self):
        import scipy.sparse as sp
        n, m, _ = self.info()
        rp, ci, cv = self.arrays()
        return sp.csr_matrix((cv, ci, rp), shape=(n, m))

    # ParMatrix::mult / residual / mult_T / mult_append (par_matrix.hpp:243-250)
    def mult(self, x, b):
        check(lib().rb_spmv(self.h, x.h, b.h))

    def residual(self, x, b, r):
        check(lib().rb_residual(self.h, x.h, b.h, r.h))

    def mult_T(self, x, b):
        check(lib().rb_spmv_T(self.h, x.h, b.h))

    def mult_append(self, x, b):
        check(lib().rb_spmv_append(self.h, x.h, b.h))

    def sort_diag_first(self):
        check(lib().rb_csr_sort_diag_first(self.h))
        return self

    def transpose(self):
        h = C.c_void_p()
        check(lib().rb_csr_transpose(self.h, C.byref(h)))
        return ParCSRMatrix(h)

    def strength(self, strength_type=Classical, theta=0.0):
        h = C.c_void_p()
        check(lib().rb_strength(self.h, int(strength_type), float(theta), C.byref(h)))
        return ParCSRMatrix(h)

    def mult_matrix(self, B):
        h = C.c_void_p()
        check(lib().rb_spgemm(self.h, B.h, C.byref(h)))
        return ParCSRMatrix(h)


def bcoo_to_bsr_arrays(n_rows, b_rows, b_cols, rows, cols, blocks):
    """Block COO -> block CSR arrays on the host, as BCOOMatrix::to_BSR does
    (core/matrix.cpp:1116-1123 with COO_to_CSR, :285-330): blocks grouped by
    block row, in the order they were added within a row.  Returns (rowptr,
    cols, blocks) with blocks of shape (nnz, b_rows, b_cols)."""
    rows = np.asarray(rows, dtype=np.int64).reshape(-1)
    cols = np.asarray(cols, dtype=np.int64).reshape(-1)
    blocks = np.asarray(blocks, dtype=np.float64).reshape(len(rows), int(b_rows), int(b_cols))
    if len(cols) != len(rows):
        raise RaptorError(-1, "rows and cols must have one entry a block")
    if rows.size and (rows.min() < 0 or rows.max() >= n_rows):
        raise RaptorError(-1, "block row index out of range")
    order = np.argsort(rows, kind="stable")
    rowptr = np.zeros(int(n_rows) + 1, np.int32)
    rowptr[1:] = np.cumsum(np.bincount(rows, minlength=int(n_rows)))
    return rowptr, cols[order].astype(np.int32), blocks[order]


def bsr_sort_diag_first(n_rows, b_rows, b_cols, rowptr, cols, blocks):
    """BSRMatrix::sort, move_diag and remove_duplicates on host block CSR
    arrays (core/matrix.cpp:588-618 sort_helper, :730-786 move_diag_helper,
    remove_duplicates_helper): a block row's blocks ordered by block column
    with the diagonal block (column == row) first, blocks whose absolute
    entries sum below 1e-16 dropped.  Blocks of one column in one row are
    summed entry by entry, in storage order; the reference's block
    append_vals (core/matrix.hpp:219-226) adds the first entries of the
    following blocks instead, so rows with repeated columns differ from it
    there.  Returns (rowptr, cols, blocks), blocks of shape (nnz, b_rows,
    b_cols)."""
    rp = np.asarray(rowptr, dtype=np.int64)
    ci = np.asarray(cols, dtype=np.int64)
    bs = int(b_rows) * int(b_cols)
    bl = np.asarray(blocks, dtype=np.float64).reshape(len(ci), bs)
    rows = np.repeat(np.arange(int(n_rows)), np.diff(rp))
    order = np.lexsort((ci, rows))                      # stable: storage order among equals
    rows, ci, bl = rows[order], ci[order], bl[order]
    if len(ci):
        first = np.ones(len(ci), bool)
        first[1:] = (rows[1:] != rows[:-1]) | (ci[1:] != ci[:-1])
        starts = np.nonzero(first)[0]
        bl = np.add.reduceat(bl, starts, axis=0)
        rows, ci = rows[starts], ci[starts]
        keep = np.abs(bl).sum(axis=1) >= 1e-16
        rows, ci, bl = rows[keep], ci[keep], bl[keep]
        order = np.lexsort((ci, ci != rows, rows))      # diagonal block first
        rows, ci, bl = rows[order], ci[order], bl[order]
    out_rp = np.zeros(int(n_rows) + 1, np.int32)
    out_rp[1:] = np.cumsum(np.bincount(rows, minlength=int(n_rows)))
    return out_rp, ci.astype(np.int32), bl.reshape(len(ci), int(b_rows), int(b_cols))


class BSRMatrix:
    """Device block CSR matrix (core/matrix.hpp:962-1060): n_rows x n_cols
    blocks of b_rows x b_cols FP64 values, int32 block indices.  Block j's
    values are the j-th b_rows x b_cols slice of the value array, row-major
    (the reference's block_vals[j][r * b_cols + c]).  Products take and give
    scalar vectors: n_cols * b_cols entries in, n_rows * b_rows out."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def from_arrays(cls, n_rows, n_cols, b_rows, b_cols, rowptr, cols, block_vals):
        """From block CSR arrays; block_vals holds nnz blocks (any shape with
        nnz * b_rows * b_cols values, block after block, row-major)."""
        rp = np.ascontiguousarray(rowptr, dtype=np.int32)
        ci = np.ascontiguousarray(cols, dtype=np.int32)
        bv = np.ascontiguousarray(block_vals, dtype=np.float64).reshape(-1)
        # the C ABI reads rowptr[n_rows] and nnz entries: refuse short arrays here
        if rp.size != int(n_rows) + 1:
            raise RaptorError(-1, "rowptr must have n_rows + 1 entries")
        if ci.size != int(rp[-1]):
            raise RaptorError(-1, "cols must have rowptr[n_rows] entries")
        if bv.size != ci.size * int(b_rows) * int(b_cols):
            raise RaptorError(-1, "block_vals must hold nnz * b_rows * b_cols values")
        if ci.size == 0:
            ci = np.zeros(1, np.int32)
            bv = np.zeros(1, np.float64)
        h = C.c_void_p()
        check(lib().rb_bsr_create(int(n_rows), int(n_cols), int(b_rows), int(b_cols), int(rp[-1]),
                                  _ptr(rp), _ptr(ci), _ptr(bv), 0, C.byref(h)))
        return cls(h)

    @classmethod
    def from_blocks(cls, n_rows, n_cols, b_rows, b_cols, rows, cols, blocks):
        """BCOOMatrix::add_value for each (rows[k], cols[k], blocks[k]), then
        to_BSR (core/matrix.cpp:1116-1123 with COO_to_CSR, :285-330): blocks
        grouped by block row, in the order they were added within a row."""
        rowptr, cols, blocks = bcoo_to_bsr_arrays(n_rows, b_rows, b_cols, rows, cols, blocks)
        return cls.from_arrays(n_rows, n_cols, b_rows, b_cols, rowptr, cols, blocks)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().rb_bsr_destroy(self.h)
            except Exception:  # noqa: BLE001
                pass
            self.h = None

    def info(self):
        r, c, br, bc, z = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int64()
        check(lib().rb_bsr_info(self.h, C.byref(r), C.byref(c), C.byref(br), C.byref(bc),
                                C.byref(z)))
        return r.value, c.value, br.value, bc.value, z.value

    @property
    def n_rows(self):
        return self.info()[0]

    @property
    def n_cols(self):
        return self.info()[1]

    @property
    def b_rows(self):
        return self.info()[2]

    @property
    def b_cols(self):
        return self.info()[3]

    @property
    def nnz(self):
        return self.info()[4]

    def arrays(self):
        """(rowptr, cols, blocks) on the host; blocks has shape (nnz, b_rows, b_cols)."""
        n, _, br, bc, z = self.info()
        rp = np.zeros(n + 1, np.int32)
        ci = np.zeros(max(z, 1), np.int32)
        bv = np.zeros(max(z * br * bc, 1), np.float64)
        check(lib().rb_bsr_download(self.h, _ptr(rp), _ptr(ci), _ptr(bv)))
        return rp, ci[:z], bv[: z * br * bc].reshape(z, br, bc)

    # Matrix::mult / mult_T / mult_append / residual (core/matrix.hpp:338-368)
    def mult(self, x, b):
        check(lib().rb_bsr_spmv(self.h, x.h, b.h))

    def mult_T(self, x, b):
        check(lib().rb_bsr_spmv_T(self.h, x.h, b.h))

    def mult_append(self, x, b):
        check(lib().rb_bsr_spmv_append(self.h, x.h, b.h))

    def residual(self, x, b, r):
        check(lib().rb_bsr_residual(self.h, x.h, b.h, r.h))

    def sort_diag_first(self):
        """BSRMatrix::sort, move_diag and remove_duplicates (see
        bsr_sort_diag_first, done on the host): a new matrix."""
        n, m, br, bc, _ = self.info()
        rp, ci, bl = self.arrays()
        rp, ci, bl = bsr_sort_diag_first(n, br, bc, rp, ci, bl)
        return BSRMatrix.from_arrays(n, m, br, bc, rp, ci, bl)

    def to_CSR(self):
        """BSRMatrix::to_CSR (core/matrix.cpp:1180-1185): the scalar matrix,
        entries with |v| > 1e-16, unsorted as the reference leaves them."""
        h = C.c_void_p()
        check(lib().rb_bsr_to_csr(self.h, C.byref(h)))
        return ParCSRMatrix(h)


# gallery ---------------------------------------------------------------------
def diffusion_stencil_2d(eps=1.0, theta=0.0):
    out = np.zeros(9)
    check(lib().rb_diffusion_stencil_2d(float(eps), float(theta), out))
    return out


def laplace_stencil_27pt():
    out = np.zeros(27)
    check(lib().rb_laplace_stencil_27pt(out))
    return out


def par_stencil_grid(stencil, grid, dim=None):
    g = np.ascontiguousarray(grid, np.int32)
    st = np.ascontiguousarray(stencil, np.float64)
    h = C.c_void_p()
    check(lib().rb_stencil_grid(st, g, int(dim or len(g)), C.byref(h)))
    return ParCSRMatrix(h)


def readParMatrix(path):
    h = C.c_void_p()
    check(lib().rb_read_petsc(str(path).encode(), C.byref(h)))
    return ParCSRMatrix(h)


def read_mm(path):
    """read_mm (gallery/matrix_market.cpp:18-76): file order within rows,
    the symmetry field ignored."""
    h = C.c_void_p()
    check(lib().rb_read_mm(str(path).encode(), C.byref(h)))
    return ParCSRMatrix(h)


def read_par_mm(path):
    """read_par_mm (gallery/par_matrix_market.cpp:18-128): symmetric files
    mirrored (each diagonal entry once), rows sorted by column."""
    h = C.c_void_p()
    check(lib().rb_read_par_mm(str(path).encode(), C.byref(h)))
    return ParCSRMatrix(h)


def write_mm(A, path):
    """write_mm / write_par_mm (gallery/matrix_market.cpp:78-105)."""
    check(lib().rb_write_mm(A.h, str(path).encode()))


write_par_mm = write_mm


def mm_read_host(path, mirror=True, sort_rows=True):
    """The MatrixMarket parser into host arrays (no device): returns
    (n_rows, n_cols, rowptr, cols, vals).  mirror=True, sort_rows=True is
    read_par_mm's matrix, False/False read_mm's."""
    m, n, z = C.c_int(), C.c_int(), C.c_int64()
    p = str(path).encode()
    check(lib().rb_mm_read_host(p, int(mirror), int(sort_rows), C.byref(m), C.byref(n),
                                C.byref(z), None, None, None))
    rp = np.zeros(m.value + 1, np.int32)
    ci = np.zeros(max(z.value, 1), np.int32)
    cv = np.zeros(max(z.value, 1), np.float64)
    check(lib().rb_mm_read_host(p, int(mirror), int(sort_rows), C.byref(m), C.byref(n),
                                C.byref(z), _ptr(rp), _ptr(ci), _ptr(cv)))
    return m.value, n.value, rp, ci[:z.value], cv[:z.value]


def mm_write_host(path, n_rows, n_cols, rowptr, cols, vals):
    """write_mm from host CSR arrays (no device)."""
    rp = np.ascontiguousarray(rowptr, np.int32)
    ci = np.ascontiguousarray(cols, np.int32)
    cv = np.ascontiguousarray(vals, np.float64)
    check(lib().rb_mm_write_host(str(path).encode(), int(n_rows), int(n_cols), int(rp[-1]),
                                 _ptr(rp), _ptr(ci) if ci.size else None,
                                 _ptr(cv) if cv.size else None))


def write_petsc(A, path):
    """Write a device matrix as a PETSc binary AIJ file (what PETSc's MatLoad
    and readParMatrix read), rows and entries in the matrix's order."""
    check(lib().rb_write_petsc(A.h, str(path).encode()))


def petsc_read_host(path):
    """readMatrix's parsing of a PETSc binary AIJ file into host arrays in
    file order (gallery/matrix_IO.cpp:24-110; no device): returns (n_rows,
    n_cols, rowptr, cols, vals)."""
    m, n, z = C.c_int(), C.c_int(), C.c_int64()
    p = str(path).encode()
    check(lib().rb_petsc_read_host(p, C.byref(m), C.byref(n), C.byref(z), None, None, None))
    rp = np.zeros(m.value + 1, np.int32)
    ci = np.zeros(max(z.value, 1), np.int32)
    cv = np.zeros(max(z.value, 1), np.float64)
    check(lib().rb_petsc_read_host(p, C.byref(m), C.byref(n), C.byref(z), _ptr(rp), _ptr(ci),
                                   _ptr(cv)))
    return m.value, n.value, rp, ci[:z.value], cv[:z.value]


def petsc_write_host(path, n_rows, n_cols, rowptr, cols, vals):
    """Write host CSR arrays as a PETSc binary AIJ file (no device)."""
    rp = np.ascontiguousarray(rowptr, np.int32)
    ci = np.ascontiguousarray(cols, np.int32)
    cv = np.ascontiguousarray(vals, np.float64)
    check(lib().rb_petsc_write_host(str(path).encode(), int(n_rows), int(n_cols), int(rp[-1]),
                                    _ptr(rp), _ptr(ci) if ci.size else None,
                                    _ptr(cv) if cv.size else None))


# setup components ---------------------------------------------------------
def split_pmis(S, weights=None):
    n = S.global_num_rows
    st = np.zeros(max(n, 1), np.int32)
    w = None if weights is None else np.ascontiguousarray(weights[:n], np.float64)
    check(lib().rb_split_pmis(S.h, _ptr(w) if w is not None else None, st))
    return st[:n]


def split(S, coarsen_type, weights=None):
    """The C/F splittings at one rank (split_rs, split_cljp, split_falgout,
    split_pmis, split_hmis of par_cf_splitting.cpp), by coarsen_t."""
    n = S.global_num_rows
    st = np.zeros(max(n, 1), np.int32)
    w = None if weights is None else np.ascontiguousarray(weights[:n], np.float64)
    check(lib().rb_split(S.h, int(coarsen_type), _ptr(w) if w is not None else None, st))
    return st[:n]


def split_rs(S):
    return split(S, RS)


def split_cljp(S, weights=None):
    return split(S, CLJP, weights)


def split_falgout(S, weights=None):
    return split(S, Falgout, weights)


def split_hmis(S, weights=None):
    return split(S, HMIS, weights)


def interpolation(A, S, states, interp_type=ModClassical, filter_threshold=0.0):
    h = C.c_void_p()
    st = np.ascontiguousarray(states, np.int32)
    check(lib().rb_interpolation(A.h, S.h, st, int(interp_type), float(filter_threshold), C.byref(h)))
    return ParCSRMatrix(h)


def direct_interpolation(A, S, states):
    return interpolation(A, S, states, Direct)


def mod_classical_interpolation(A, S, states):
    return interpolation(A, S, states, ModClassical)


def extended_interpolation(A, S, states, filter_threshold=0.3):
    return interpolation(A, S, states, Extended, filter_threshold)


def rap(A, P, diag_first=True):
    h = C.c_void_p()
    check(lib().rb_rap(A.h, P.h, 1 if diag_first else 0, C.byref(h)))
    return ParCSRMatrix(h)


def mis2(S, weights=None):
    """mis2 (aggregation/par_mis.cpp:204-645): 1 = root, 0 = not a root."""
    n = S.global_num_rows
    st = np.zeros(max(n, 1), np.int32)
    w = None if weights is None else np.ascontiguousarray(weights[:n], np.float64)
    check(lib().rb_mis2(S.h, _ptr(w) if w is not None else None, st))
    return st[:n]


def aggregate(A, S, states, rand_vals=None):
    """aggregate (aggregation/par_aggregate.cpp:5-185) -> (n_aggs, aggregates);
    aggregates hold each row's root row index, -1 when unaggregated."""
    n = S.global_num_rows
    st = np.ascontiguousarray(states, np.int32)
    agg = np.zeros(max(n, 1), np.int32)
    r = None if rand_vals is None else np.ascontiguousarray(rand_vals[:n], np.float64)
    na = C.c_int()
    check(lib().rb_aggregate(A.h, S.h, st, _ptr(r) if r is not None else None, agg, C.byref(na)))
    return na.value, agg[:n]


def fit_candidates(n, n_aggs, aggregates, B):
    """fit_candidates with one candidate (aggregation/par_candidates.cpp:6-216)
    -> (T, R)."""
    agg = np.ascontiguousarray(aggregates, np.int32)
    Bv = np.ascontiguousarray(B[:n], np.float64)
    R = np.zeros(max(n_aggs, 1), np.float64)
    h = C.c_void_p()
    check(lib().rb_fit_candidates(int(n), int(n_aggs), agg, Bv, R, C.byref(h)))
    return ParCSRMatrix(h), R[:n_aggs]


def jacobi_prolongation(A, T, omega=4.0 / 3.0, num_smooth_steps=1):
    """jacobi_prolongation (aggregation/par_prolongation.cpp:7-104)."""
    h = C.c_void_p()
    check(lib().rb_jacobi_prolongation(A.h, T.h, float(omega), int(num_smooth_steps), C.byref(h)))
    return ParCSRMatrix(h)


# multilevel ---------------------------------------------------------------
class ParMultilevel:
    """ParMultilevel (multilevel/par_multilevel.hpp:75-659) on the device."""

    _FIELDS = ("strong_threshold", "relax_weight", "num_smooth_sweeps", "max_coarse",
               "max_levels", "max_iterations", "solve_tol", "interp_filter")
    _EXTRA = ("precision", "jacobi_compat", "seed_offset", "relax_type", "strength_type",
              "interp_type", "fuse_coarse", "use_graphs", "const_coef", "coarsen_type", "num_variables",
              "prolong_weight",
              "prolong_smooth_steps", "solver")

    def __init__(self, strong_threshold=0.0, strength_type=Classical, relax_type=SOR):
        self.opts = AmgOpts()
        lib().rb_amg_default_opts(C.byref(self.opts))
        self.opts.strong_threshold = strong_threshold
        self.opts.strength_type = strength_type
        self.opts.relax_type = relax_type
        self.h = None
        self.weights = None
        self.residuals = []
        self.store_residuals = True

    def __getattr__(self, name):
        if name in ParMultilevel._FIELDS or name in ParMultilevel._EXTRA:
            return getattr(self.__dict__["opts"], name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in ParMultilevel._FIELDS or name in ParMultilevel._EXTRA:
            setattr(self.opts, name, value)
        else:
            object.__setattr__(self, name, value)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().rb_amg_destroy(self.h)
            except Exception:  # noqa: BLE001
                pass
            self.h = None

    def setup(self, A):
        if self.h:
            lib().rb_amg_destroy(self.h)
            self.h = None
        h = C.c_void_p()
        w = None
        if self.weights is not None:
            self._w = np.ascontiguousarray(self.weights, np.float64)
            w = _ptr(self._w)
        check(lib().rb_amg_setup(A.h, C.byref(self.opts), w, C.byref(h)))
        self.h = h
        self.A = A

    @property
    def num_levels(self):
        n = C.c_int()
        check(lib().rb_amg_num_levels(self.h, C.byref(n)))
        return n.value

    def level_info(self, l):
        n, za, zp = C.c_int(), C.c_int64(), C.c_int64()
        check(lib().rb_amg_level_info(self.h, l, C.byref(n), C.byref(za), C.byref(zp)))
        return n.value, za.value, zp.value

    def level_matrix(self, l, which="A"):
        h = C.c_void_p()
        check(lib().rb_amg_level_matrix(self.h, l, {"A": 0, "P": 1, "R": 2}[which], C.byref(h)))
        return ParCSRMatrix(h)

    def level_states(self, l):
        n = self.level_info(l)[0]
        st = np.zeros(max(n, 1), np.int32)
        check(lib().rb_amg_level_states(self.h, l, st))
        return st[:n]

    def cycle(self, x, b, level=0):
        check(lib().rb_amg_cycle(self.h, x.h, b.h))

    def solve(self, x, b):
        cap = self.opts.max_iterations + 1
        hist = np.zeros(cap)
        it = C.c_int()
        rc = lib().rb_amg_solve(self.h, x.h, b.h, C.byref(it), _ptr(hist), cap)
        self.residuals = list(hist[: it.value + 1])
        if rc not in (0, -5):
            check(rc)
        return it.value

    def get_residuals(self):
        return self.residuals

    def cycle_block(self, X, B, k):
        """X = M B for k interleaved columns (one V-cycle from a zero guess)."""
        check(lib().rb_amg_cycle_block(self.h, X.h, B.h, int(k)))

    def cycle_profile(self):
        """Milliseconds per level: rows [pre, residual, restrict, prolong, post, coarse]."""
        L = self.num_levels
        ms = np.zeros(8 * L)
        n = C.c_int()
        check(lib().rb_amg_cycle_profile(self.h, _ptr(ms), 8 * L, C.byref(n)))
        return ms.reshape(L, 8)[:, :6]

    def time_operator(self, level, op, reps=20):
        out = C.c_double()
        check(lib().rb_amg_time_operator(self.h, int(level), int(op), int(reps), C.byref(out)))
        return out.value

    @property
    def setup_seconds(self):
        out = C.c_double()
        check(lib().rb_amg_setup_seconds(self.h, C.byref(out)))
        return out.value

    def level_lanes(self, l):
        a, p, r = C.c_int(), C.c_int(), C.c_int()
        check(lib().rb_amg_level_lanes(self.h, l, C.byref(a), C.byref(p), C.byref(r)))
        return a.value, p.value, r.value

    def level_storage(self, l):
        """Number of stored diagonals of A_l (sliced layout), 0 for CSR."""
        nd = C.c_int()
        check(lib().rb_amg_level_storage(self.h, l, C.byref(nd)))
        return nd.value

    def level_const_coef(self, l):
        """0: A_l's values are read; 1: its diagonals have constant
        coefficients and the cycle reads a mask a row instead; 2: in
        addition it is a stencil on a box and the cycle stages x in shared
        memory, reading no mask (see the C ABI)."""
        f = C.c_int()
        check(lib().rb_amg_level_const_coef(self.h, l, C.byref(f)))
        return int(f.value)

    def level_fused_first(self, l):
        """True when level l's first sweep runs fused with its residual."""
        f = C.c_int()
        check(lib().rb_amg_level_fused_first(self.h, l, C.byref(f)))
        return bool(f.value)

    def tail_timings(self):
        """Cycle ms measured when the tail start was picked (see the C ABI)."""
        c = C.c_int()
        buf = np.zeros(64)
        check(lib().rb_amg_tail_timings(self.h, buf, 64, C.byref(c)))
        return [float(v) for v in buf[: min(c.value, 64)]]

    def tail_info(self):
        """(start level of the one-launch cluster tail or -1, its CTAs)."""
        f, c = C.c_int(), C.c_int()
        check(lib().rb_amg_tail_info(self.h, C.byref(f), C.byref(c)))
        return f.value, c.value

    def print_hierarchy(self):
        print("Num Levels = %d" % self.num_levels)
        print("A\tNRow\tNCol\tNNZ")
        for l in range(self.num_levels):
            n, za, _ = self.level_info(l)
            print("%d\t%d\t%d\t%d" % (l, n, n, za))


class ParRugeStubenSolver(ParMultilevel):
    """ParRugeStubenSolver (ruge_stuben/par_ruge_stuben_solver.hpp:12-170)."""

    def __init__(self, strong_threshold=0.0, coarsen_type=RS, interp_type=Direct,
                 strength_type=Classical, relax_type=SOR):
        super().__init__(strong_threshold, strength_type, relax_type)
        if coarsen_type not in (RS, CLJP, Falgout, PMIS, HMIS):
            raise RaptorError(-1, "coarsening must be RS, CLJP, Falgout, PMIS or HMIS")
        self.opts.coarsen_type = coarsen_type
        if interp_type not in (Direct, ModClassical, Extended):
            raise RaptorError(-1, "interpolation must be Direct, ModClassical or Extended")
        self.opts.interp_type = interp_type


class ParSmoothedAggregationSolver(ParMultilevel):
    """ParSmoothedAggregationSolver
    (aggregation/par_smoothed_aggregation_solver.hpp:13-136): symmetric
    strength, mis2 aggregation, one all-ones candidate, Jacobi-smoothed
    tentative prolongator, Galerkin coarse operators."""

    def __init__(self, strong_threshold=0.0, agg_type=MIS, prolong_type=JacobiProlongation,
                 strength_type=Symmetric, relax_type=SOR, prolong_smooth_steps=1,
                 prolong_weight=4.0 / 3):
        super().__init__(strong_threshold, strength_type, relax_type)
        if agg_type != MIS or prolong_type != JacobiProlongation:
            raise RaptorError(-1, "only MIS aggregation with Jacobi prolongation exists")
        self.opts.solver = 1
        self.opts.prolong_smooth_steps = prolong_smooth_steps
        self.opts.prolong_weight = prolong_weight


class Batch:
    """An uneven batch of independent systems solved together: each matrix
    gets the hierarchy a standalone setup would build, and every V-cycle
    operation runs once for all systems (rb_batch_* in the C ABI).  Vectors
    are the systems' vectors concatenated (`offsets`)."""

    def __init__(self, matrices, ml=None):
        self.matrices = list(matrices)
        opts = ml.opts if ml is not None else None
        if opts is None:
            opts = AmgOpts()
            lib().rb_amg_default_opts(C.byref(opts))
        arr = (C.c_void_p * len(self.matrices))(*[m.h.value for m in self.matrices])
        h = C.c_void_p()
        check(lib().rb_batch_setup(len(self.matrices), arr, C.byref(opts), C.byref(h)))
        self.h = h
        n = len(self.matrices)
        self.offsets = np.zeros(n + 1, np.int64)
        self.levels = np.zeros(n, np.int32)
        check(lib().rb_batch_offsets(self.h, self.offsets.ctypes.data, self.levels.ctypes.data))
        self.n_sys = n
        self.total_rows = int(self.offsets[-1])

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().rb_batch_destroy(self.h)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self.h = None

    def cycle(self, x, b):
        check(lib().rb_batch_cycle(self.h, x.h, b.h))

    @property
    def host_waits(self):
        """Host waits of the last pcg (one per launch of its device loop)."""
        w = C.c_int()
        check(lib().rb_batch_host_waits(self.h, C.byref(w)))
        return w.value

    def pcg(self, x, b, tol=1e-8, max_iter=-1):
        """Per-system PCG to tol (true relative residual); returns
        (status, iters[n_sys], relres[n_sys])."""
        iters = np.zeros(self.n_sys, np.int32)
        relres = np.zeros(self.n_sys, np.float64)
        rc = lib().rb_batch_pcg(self.h, x.h, b.h, float(tol), int(max_iter), iters, relres)
        if rc not in (0, -5):
            check(rc)
        return rc, iters, relres


# Krylov -------------------------------------------------------------------
def _hist_call(fn, cap):
    hist = np.zeros(cap)
    nh = C.c_int()
    rc = fn(hist, nh)
    return rc, list(hist[: min(nh.value, cap)])


def PCG(A, ml, x, b, res, tol=1e-5, max_iter=-1, mode=PCG_REFERENCE):
    """krylov/par_cg.cpp:121-263; appends the history to `res`."""
    cap = max(max_iter, 0) + 2 if max_iter > 0 else (int(1.3 * A.global_num_rows) + 4)
    cap = min(cap, 1 << 20)
    rc, h = _hist_call(lambda hist, nh: lib().rb_pcg(A.h, ml.h, x.h, b.h, float(tol), int(max_iter),
                                                     int(mode), _ptr(hist), cap, C.byref(nh)), cap)
    res.extend(h)
    if rc not in (0, -5):
        check(rc)
    return rc


def PCG_block(A, ml, X, B, k, tol=1e-8, max_iter=-1):
    """k right-hand sides over one hierarchy: X, B are ParVectors of n * k
    entries, columns interleaved by row.  Returns (status, iters[k], relres[k])
    with each column's iterations and final true relative residual."""
    iters = np.zeros(max(k, 1), np.int32)
    relres = np.zeros(max(k, 1), np.float64)
    rc = lib().rb_pcg_block(A.h, ml.h, X.h, B.h, int(k), float(tol), int(max_iter), iters, relres)
    if rc not in (0, -5):
        check(rc)
    return rc, iters[:k], relres[:k]


def CG(A, x, b, res, tol=1e-5, max_iter=-1):
    cap = max(max_iter, 0) + 2 if max_iter > 0 else (int(1.3 * A.global_num_rows) + 4)
    cap = min(cap, 1 << 20)
    rc, h = _hist_call(lambda hist, nh: lib().rb_cg(A.h, x.h, b.h, float(tol), int(max_iter),
                                                    _ptr(hist), cap, C.byref(nh)), cap)
    res.extend(h)
    if rc not in (0, -5):
        check(rc)
    return rc


def BiCGStab(A, x, b, res, tol=1e-5, max_iter=-1):
    cap = max(max_iter, 0) + 2 if max_iter > 0 else (int(1.3 * A.global_num_rows) + 4)
    cap = min(cap, 1 << 20)
    rc, h = _hist_call(lambda hist, nh: lib().rb_bicgstab(A.h, None, x.h, b.h, float(tol),
                                                          int(max_iter), _ptr(hist), cap,
                                                          C.byref(nh)), cap)
    res.extend(h)
    if rc not in (0, -5):
        check(rc)
    return rc


def Pre_BiCGStab(A, x, b, ml, res, tol=1e-5, max_iter=-1):
    cap = max(max_iter, 0) + 2 if max_iter > 0 else (int(1.3 * A.global_num_rows) + 4)
    cap = min(cap, 1 << 20)
    rc, h = _hist_call(lambda hist, nh: lib().rb_bicgstab(A.h, ml.h, x.h, b.h, float(tol),
                                                          int(max_iter), _ptr(hist), cap,
                                                          C.byref(nh)), cap)
    res.extend(h)
    if rc not in (0, -5):
        check(rc)
    return rc


def launch_count():
    out = C.c_int64()
    check(lib().rb_launch_count(C.byref(out)))
    return out.value


def init(device=0):
    check(lib().rb_init(int(device)))


def set_stream(cuda_stream):
    """Order all later library calls on a caller's CUDA stream (its handle as
    an integer; 0 = the library's own stream)."""
    check(lib().rb_set_stream(C.c_void_p(int(cuda_stream) or None)))


def synchronize():
    """Wait for all work queued on the library stream."""
    check(lib().rb_synchronize())


def version():
    return lib().rb_version().decode()


from . import autograd  # noqa: E402,F401  (torch is imported only when used)
