// bsr.cuh -- block CSR (BSR) products and expansion, one scalar row (or
// column) at a time.
//
// BSRMatrix (core/matrix.hpp:962-1060): n_block_rows x n_block_cols blocks of
// b_rows x b_cols values; rowptr / cols index blocks, and block j's values
// sit at vals[j * b_rows * b_cols], row-major inside the block (the
// reference keeps one heap array a block, block_vals[j][r * b_cols + c]).
// Scalar row `row` is row r = row % b_rows of block row i = row / b_rows.
//
// Every function keeps the reference's order of operations, so a build
// without contracted multiply-adds (nvcc -fmad=false, g++ -ffp-contract=off)
// gives the reference's results bit for bit:
//   * product (BSR_spmv, util/linalg/spmv.cpp:121-148): a scalar row summed
//     from zero over the block row's blocks in storage order, the columns of
//     a block in order;
//   * append (BSR_append with the block Matrix::append, spmv.cpp:105-119,
//     core/matrix.hpp:287-298): the same products added to b[row] one after
//     another;
//   * residual (BSRMatrix::spmv_residual, spmv.cpp:363-368, with the block
//     append_neg, matrix.hpp:313-324): r = b, then each product subtracted;
//   * transposed product (Matrix::mult_T, matrix.hpp:342-348, with the block
//     append_T, matrix.hpp:299-312): b zeroed, then for block rows in
//     increasing order, blocks in storage order, block rows r in order,
//     b[col] += block[r][c] * x[i * b_rows + r].  Here one thread owns one
//     scalar column and walks a transposed map of the block pattern whose
//     rows list (source block row, source block) in that same order;
//   * expansion (BSR_to_CSR, core/matrix.cpp:358-395): scalar row by scalar
//     row, the row's blocks in storage order, the block's columns in order,
//     keeping values with |v| > 1e-16 (zero_tol, core/types.hpp:26).
//
// The same functions run in the CUDA kernels (bsr.cu) and in a host build
// that tests them against the CPU restatement.
#pragma once

#include <math.h>
#include <stddef.h>

#include <vector>

#ifndef RB_HD
#if defined(__CUDACC__)
#define RB_HD __host__ __device__
#else
#define RB_HD
#endif
#endif

namespace rb {

constexpr double kBsrZeroTol = 1e-16;   // zero_tol, core/types.hpp:26

enum BsrRowOp { kBsrMult = 0, kBsrAppend = 1, kBsrResidual = 2 };

// Scalar row `row`: start + (or -, for the residual) the row of A x.
template <int OP>
RB_HD inline double bsr_row(int row, int br, int bc, const int* rowptr, const int* cols,
                            const double* vals, const double* x, double start) {
    const int i = row / br, r = row - i * br;
    const size_t bs = (size_t)br * bc;
    double acc = start;
    for (int j = rowptr[i]; j < rowptr[i + 1]; j++) {
        const double* blk = vals + (size_t)j * bs + (size_t)r * bc;
        const double* xx = x + (size_t)cols[j] * bc;
#if defined(__CUDA_ARCH__)
        // even block width: a block row and its x slice start on 16-byte
        // boundaries (cudaMalloc'd arrays), so they load as double2 pairs;
        // the products are added in the same order as below
        if ((bc & 1) == 0) {
            for (int c = 0; c < bc; c += 2) {
                const double2 v = *reinterpret_cast<const double2*>(blk + c);
                const double2 w = *reinterpret_cast<const double2*>(xx + c);
                if (OP == kBsrResidual) {
                    acc -= v.x * w.x;
                    acc -= v.y * w.y;
                } else {
                    acc += v.x * w.x;
                    acc += v.y * w.y;
                }
            }
            continue;
        }
#endif
        for (int c = 0; c < bc; c++) {
            if (OP == kBsrResidual)
                acc -= blk[c] * xx[c];
            else
                acc += blk[c] * xx[c];
        }
    }
    return acc;
}

// Scalar column `col` of A^T x, through the transposed block pattern: block
// column q's entries k in [trowptr[q], trowptr[q+1]) name the source block
// row trows[k] and the source block tsrc[k].
RB_HD inline double bsr_col_T(int col, int br, int bc, const int* trowptr, const int* trows,
                              const int* tsrc, const double* vals, const double* x) {
    const int q = col / bc, c = col - q * bc;
    const size_t bs = (size_t)br * bc;
    double acc = 0.0;
    for (int k = trowptr[q]; k < trowptr[q + 1]; k++) {
        const double* blk = vals + (size_t)tsrc[k] * bs + c;
        const double* xx = x + (size_t)trows[k] * br;
        for (int r = 0; r < br; r++) acc += blk[(size_t)r * bc] * xx[r];
    }
    return acc;
}

// The transposed block pattern (host): a stable counting sort of the blocks
// by block column, so block column q lists (block row i, block j) for i
// increasing and, inside a block row, j in storage order -- the order the
// reference's scatter adds them.  trowptr has nbc + 1 entries, trows and tsrc
// rowptr[nbr].  rowptr and cols must be valid (monotone, columns < nbc).
inline void bsr_transpose_pattern(int nbr, int nbc, const int* rowptr, const int* cols,
                                  int* trowptr, int* trows, int* tsrc) {
    for (int q = 0; q <= nbc; q++) trowptr[q] = 0;
    for (int j = 0; j < rowptr[nbr]; j++) trowptr[cols[j] + 1]++;
    for (int q = 0; q < nbc; q++) trowptr[q + 1] += trowptr[q];
    std::vector<int> next(trowptr, trowptr + nbc);
    for (int i = 0; i < nbr; i++)
        for (int j = rowptr[i]; j < rowptr[i + 1]; j++) {
            const int k = next[cols[j]]++;
            trows[k] = i;
            tsrc[k] = j;
        }
}

// Entries scalar row `row` keeps when expanded to CSR.
RB_HD inline int bsr_csr_row_count(int row, int br, int bc, const int* rowptr,
                                   const double* vals) {
    const int i = row / br, r = row - i * br;
    const size_t bs = (size_t)br * bc;
    int n = 0;
    for (int j = rowptr[i]; j < rowptr[i + 1]; j++) {
        const double* blk = vals + (size_t)j * bs + (size_t)r * bc;
        for (int c = 0; c < bc; c++) n += fabs(blk[c]) > kBsrZeroTol;
    }
    return n;
}

// Writes scalar row `row`'s entries from position `first` of the CSR arrays.
RB_HD inline void bsr_csr_row_fill(int row, int br, int bc, const int* rowptr, const int* cols,
                                   const double* vals, int first, int* out_cols,
                                   double* out_vals) {
    const int i = row / br, r = row - i * br;
    const size_t bs = (size_t)br * bc;
    int k = first;
    for (int j = rowptr[i]; j < rowptr[i + 1]; j++) {
        const double* blk = vals + (size_t)j * bs + (size_t)r * bc;
        for (int c = 0; c < bc; c++) {
            const double v = blk[c];
            if (fabs(v) > kBsrZeroTol) {
                out_cols[k] = cols[j] * bc + c;
                out_vals[k] = v;
                k++;
            }
        }
    }
}

}  // namespace rb
