// bsr.cu -- block CSR (BSRMatrix) products and expansion to CSR.
//
// One thread a scalar row (a scalar column for the transposed product): a
// thread walks its block row's blocks and reads one b_cols-wide row of each,
// so the b_rows threads of a block row read each block between them.  The
// products are bound by HBM: 8 B a stored value plus 4 B a block index and
// the gathered x.  Built with -fmad=false, so every product and sum rounds
// separately, in the reference's order (bsr.cuh), and results are the
// reference's bit for bit.
#include <climits>
#include <memory>
#include <vector>

#include "bsr.cuh"
#include "rb_internal.cuh"

namespace rb {

namespace {

constexpr int kBsrBlock = 256;
// six resident blocks an SM (1536 threads): 40 registers; the append and
// residual forms keep one 8-byte value on the stack
constexpr int kBsrMinBlocks = 6;

template <int OP>
__global__ void __launch_bounds__(kBsrBlock, kBsrMinBlocks)
    k_bsr_rows(int n, int br, int bc, const int* __restrict__ rowptr, const int* __restrict__ cols,
               const double* __restrict__ vals, const double* __restrict__ x, const double* b,
               double* y) {
    const long row = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    const double start = OP == kBsrMult ? 0.0 : b[row];
    y[row] = bsr_row<OP>(row, br, bc, rowptr, cols, vals, x, start);
}

__global__ void __launch_bounds__(kBsrBlock, kBsrMinBlocks)
    k_bsr_cols_T(int n, int br, int bc, const int* __restrict__ trowptr,
                 const int* __restrict__ trows, const int* __restrict__ tsrc,
                 const double* __restrict__ vals, const double* __restrict__ x,
                 double* __restrict__ y) {
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= n) return;
    y[col] = bsr_col_T(col, br, bc, trowptr, trows, tsrc, vals, x);
}

__global__ void __launch_bounds__(kBsrBlock, kBsrMinBlocks)
    k_bsr_csr_count(int n, int br, int bc, const int* __restrict__ rowptr,
                    const double* __restrict__ vals, int* __restrict__ counts) {
    const long row = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    counts[row] = bsr_csr_row_count(row, br, bc, rowptr, vals);
}

__global__ void __launch_bounds__(kBsrBlock, kBsrMinBlocks)
    k_bsr_csr_fill(int n, int br, int bc, const int* __restrict__ rowptr,
                   const int* __restrict__ cols, const double* __restrict__ vals,
                   const int* __restrict__ out_rowptr, int* __restrict__ out_cols,
                   double* __restrict__ out_vals) {
    const long row = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    bsr_csr_row_fill(row, br, bc, rowptr, cols, vals, out_rowptr[row], out_cols, out_vals);
}

// The transposed block pattern, built on the host (bsr_transpose_pattern)
// from the handle's rowptr and cols and kept on the handle.
void build_tmap(rb_bsr_s& A) {
    const int nbr = A.n_block_rows, nbc = A.n_block_cols;
    const size_t nnz = (size_t)A.nnz;
    std::vector<int> rp((size_t)nbr + 1), ci(nnz);
    A.rowptr.download(rp.data(), rp.size());
    A.cols.download(ci.data(), nnz);
    RB_CUDA(cudaStreamSynchronize(stream()));
    // device-created matrices were not checked at creation
    RB_REQUIRE(rp[0] == 0 && (size_t)rp[nbr] == nnz, "block rowptr does not span the blocks");
    for (int i = 0; i < nbr; i++) RB_REQUIRE(rp[i] <= rp[(size_t)i + 1], "block rowptr is not monotone");
    for (size_t j = 0; j < nnz; j++)
        RB_REQUIRE(ci[j] >= 0 && ci[j] < nbc, "block column index out of range");
    std::vector<int> trp((size_t)nbc + 1), trows(nnz > 0 ? nnz : 1), tsrc(nnz > 0 ? nnz : 1);
    bsr_transpose_pattern(nbr, nbc, rp.data(), ci.data(), trp.data(), trows.data(), tsrc.data());
    auto m = std::make_unique<TransposeMap>();
    m->rowptr.alloc(trp.size());
    m->rows.alloc(trows.size());
    m->src.alloc(tsrc.size());
    m->rowptr.upload(trp.data(), trp.size());
    m->rows.upload(trows.data(), nnz);
    m->src.upload(tsrc.data(), nnz);
    RB_CUDA(cudaStreamSynchronize(stream()));
    A.tmap = std::move(m);
}

}  // namespace

void bsr_apply(const rb_bsr_s& A, int op, const double* x, const double* b, double* y) {
    const int n = A.n_block_rows * A.b_rows;
    if (n == 0) return;
    const unsigned grid = grid_for(n, kBsrBlock);
    const int br = A.b_rows, bc = A.b_cols;
    switch (op) {
        case kBsrMult:
            k_bsr_rows<kBsrMult><<<grid, kBsrBlock, 0, stream()>>>(
                n, br, bc, A.rowptr.get(), A.cols.get(), A.vals.get(), x, b, y);
            break;
        case kBsrAppend:
            k_bsr_rows<kBsrAppend><<<grid, kBsrBlock, 0, stream()>>>(
                n, br, bc, A.rowptr.get(), A.cols.get(), A.vals.get(), x, b, y);
            break;
        case kBsrResidual:
            k_bsr_rows<kBsrResidual><<<grid, kBsrBlock, 0, stream()>>>(
                n, br, bc, A.rowptr.get(), A.cols.get(), A.vals.get(), x, b, y);
            break;
        default:
            RB_REQUIRE(false, "unknown block product");
    }
    RB_CHECK_LAUNCH();
}

void bsr_spmv_T(rb_bsr_s& A, const double* x, double* y) {
    if (!A.tmap) build_tmap(A);
    const int n = A.n_block_cols * A.b_cols;
    if (n == 0) return;
    k_bsr_cols_T<<<grid_for(n, kBsrBlock), kBsrBlock, 0, stream()>>>(
        n, A.b_rows, A.b_cols, A.tmap->rowptr.get(), A.tmap->rows.get(), A.tmap->src.get(),
        A.vals.get(), x, y);
    RB_CHECK_LAUNCH();
}

rb_csr_s* bsr_to_csr(const rb_bsr_s& A) {
    const int n = A.n_block_rows * A.b_rows;
    const int m = A.n_block_cols * A.b_cols;
    DevArray<int> counts(n > 0 ? (size_t)n : 1);
    if (n) {
        k_bsr_csr_count<<<grid_for(n, kBsrBlock), kBsrBlock, 0, stream()>>>(
            n, A.b_rows, A.b_cols, A.rowptr.get(), A.vals.get(), counts.get());
        RB_CHECK_LAUNCH();
    }
    DevArray<int> rp((size_t)n + 1);
    const long long nnz = exclusive_scan(counts.get(), rp.get(), n);
    std::unique_ptr<rb_csr_s> C(new_csr(n, m, nnz));
    C->rowptr = std::move(rp);
    if (n && nnz) {
        k_bsr_csr_fill<<<grid_for(n, kBsrBlock), kBsrBlock, 0, stream()>>>(
            n, A.b_rows, A.b_cols, A.rowptr.get(), A.cols.get(), A.vals.get(), C->rowptr.get(),
            C->cols.get(), C->vals.get());
        RB_CHECK_LAUNCH();
    }
    RB_CUDA(cudaStreamSynchronize(stream()));
    return C.release();
}

}  // namespace rb
