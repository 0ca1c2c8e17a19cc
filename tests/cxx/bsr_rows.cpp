// Host build of the per-row block CSR code that the CUDA kernels run
// (raptor_b200/csrc/bsr.cuh), for a CPU test against the restatement and the
// reference: one loop iteration per thread of the kernels, in any order.
#include <vector>

#include "bsr.cuh"

extern "C" void bsr_rows_apply(int op, int nbr, int br, int bc, const int* rp, const int* ci,
                               const double* v, const double* x, const double* b, double* y) {
    const int n = nbr * br;
    for (int row = n - 1; row >= 0; row--) {   // any order: rows are independent
        switch (op) {
            case rb::kBsrMult: y[row] = rb::bsr_row<rb::kBsrMult>(row, br, bc, rp, ci, v, x, 0.0); break;
            case rb::kBsrAppend:
                y[row] = rb::bsr_row<rb::kBsrAppend>(row, br, bc, rp, ci, v, x, b[row]);
                break;
            default:
                y[row] = rb::bsr_row<rb::kBsrResidual>(row, br, bc, rp, ci, v, x, b[row]);
        }
    }
}

extern "C" void bsr_cols_T(int nbr, int nbc, int br, int bc, const int* rp, const int* ci,
                           const double* v, const double* x, double* y) {
    const int nnz = rp[nbr];
    std::vector<int> trp(nbc + 1), trows(nnz + 1), tsrc(nnz + 1);
    rb::bsr_transpose_pattern(nbr, nbc, rp, ci, trp.data(), trows.data(), tsrc.data());
    for (int col = nbc * bc - 1; col >= 0; col--)
        y[col] = rb::bsr_col_T(col, br, bc, trp.data(), trows.data(), tsrc.data(), v, x);
}

// Count pass, prefix sum, fill pass, as bsr_to_csr launches them.
extern "C" int bsr_csr_count(int nbr, int br, int bc, const int* rp, const double* v, int* out_rp) {
    const int n = nbr * br;
    out_rp[0] = 0;
    for (int row = 0; row < n; row++)
        out_rp[row + 1] = out_rp[row] + rb::bsr_csr_row_count(row, br, bc, rp, v);
    return out_rp[n];
}

extern "C" void bsr_csr_fill(int nbr, int br, int bc, const int* rp, const int* ci,
                             const double* v, const int* out_rp, int* out_ci, double* out_v) {
    for (int row = nbr * br - 1; row >= 0; row--)
        rb::bsr_csr_row_fill(row, br, bc, rp, ci, v, out_rp[row], out_ci, out_v);
}
