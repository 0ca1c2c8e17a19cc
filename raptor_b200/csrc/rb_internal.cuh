// rb_internal.cuh -- handle types behind the C ABI and shared declarations.
#pragma once

#include <memory>
#include <vector>

#include "rb_common.cuh"

namespace rb {
// The pattern of A^T with, for each of its entries, the position in A's
// value array it comes from: rows of A^T list source rows in increasing
// order.  Built on the first transposed product and kept on the handle, so
// later products gather A's current values through it (values may change
// between calls, the pattern may not).
struct TransposeMap {
    DevArray<int> rowptr, rows, src;
};
}  // namespace rb

struct rb_csr_s {
    int n_rows = 0, n_cols = 0;
    long long nnz = 0;
    rb::DevArray<int> rowptr, cols;
    rb::DevArray<double> vals;
    std::unique_ptr<rb::TransposeMap> tmap;  // lazily built by spmv_T64
    int lanes = 0;  // row-kernel schedule of the public products (timed on first use)
};

struct rb_batch_s;

// Block CSR: block j's values at vals[j * b_rows * b_cols], row-major.
struct rb_bsr_s {
    int n_block_rows = 0, n_block_cols = 0, b_rows = 1, b_cols = 1;
    long long nnz = 0;  // blocks
    rb::DevArray<int> rowptr, cols;
    rb::DevArray<double> vals;
    // block pattern of A^T (rows: block columns; entries: source block row
    // and source block), built by the first transposed product
    std::unique_ptr<rb::TransposeMap> tmap;
};

struct rb_vec_s {
    int n = 0;
    rb::DevArray<double> v;
};

namespace rb {

// Non-owning view of a CSR matrix with values of type T.
template <typename T>
struct CsrView {
    int n_rows = 0, n_cols = 0;
    long long nnz = 0;
    const int* rowptr = nullptr;
    const int* cols = nullptr;
    const T* vals = nullptr;
};

inline CsrView<double> view(const rb_csr_s& A) {
    CsrView<double> v;
    v.n_rows = A.n_rows; v.n_cols = A.n_cols; v.nnz = A.nnz;
    v.rowptr = A.rowptr.get(); v.cols = A.cols.get(); v.vals = A.vals.get();
    return v;
}

rb_csr_s* new_csr(int n_rows, int n_cols, long long nnz);
// CSR arrays on the host (file I/O)
struct HostCsr {
    int n_rows = 0, n_cols = 0;
    std::vector<int> rowptr, cols;
    std::vector<double> vals;
};
// MatrixMarket coordinate file -> host CSR: mirror stores (j, i) for the
// off-diagonal entries of symmetric / skew-symmetric files, sort_rows sorts
// each row by column (stable); otherwise file order within a row (mmio.cu)
HostCsr mm_parse(const char* path, bool mirror, bool sort_rows);
// PETSc binary AIJ file <-> host CSR, rows and entries in file order (mmio.cu)
HostCsr petsc_parse(const char* path);
void petsc_write(const char* path, int n_rows, int n_cols, long long nnz, const int* rowptr,
                 const int* cols, const double* vals);
void mm_write(const char* path, int n_rows, int n_cols, long long nnz, const int* rowptr,
              const int* cols, const double* vals);
rb_csr_s* clone_csr(const rb_csr_s& M);
// Sort every row by column and move the diagonal to the front.
void sort_rows_diag_first(rb_csr_s& A, bool diag_first);
// Transpose; rows of the result list source rows in increasing order.
rb_csr_s* transpose(const rb_csr_s& A);
// Exclusive scan of n ints into out (n+1 entries, out[n] = total); returns total.
long long exclusive_scan(const int* in, int* out, int n);
// Sum of n doubles, deterministic (fixed two-stage tree).
void dot_async(const double* a, const double* b, int n, double* result_dev);

// SpMV family on FP64 CSR (C ABI primitives); lanes 0 picks the row
// schedule from the mean row length.
void spmv64(const CsrView<double>& A, const double* x, double* y, int lanes = 0);
void residual64(const CsrView<double>& A, const double* x, const double* b, double* r,
                int lanes = 0);
void spmv_append64(const CsrView<double>& A, const double* x, double* y, int lanes = 0);
// The fastest row schedule for a handle's products, timed once on x (the
// handle keeps it).
int handle_lanes(rb_csr_s& A, const double* x);
// y = A^T x through the handle's cached transpose map (built on first use).
void spmv_T64(rb_csr_s& A, const double* x, double* y);

// Block CSR products and expansion (bsr.cu).  op: kBsrMult (y = A x, b
// unused), kBsrAppend (y = b + A x, b may be y), kBsrResidual (y = b - A x).
void bsr_apply(const rb_bsr_s& A, int op, const double* x, const double* b, double* y);
// y = A^T x (builds A.tmap on first use).
void bsr_spmv_T(rb_bsr_s& A, const double* x, double* y);
// Scalar CSR of A, entries with |v| > 1e-16, in the reference's order.
rb_csr_s* bsr_to_csr(const rb_bsr_s& A);

// Setup components (setup.cu).
// vars (the unknown-based systems form, num_variables > 1; NULL otherwise):
// each row's variable; classical strength and ModClassical / Extended
// interpolation couple only rows of one variable (the reference's symmetric
// strength and Direct ignore it)
rb_csr_s* strength(const rb_csr_s& A, int kind, double theta, const int* vars = nullptr);
// the finest level's variable list (row i: i % nv), and the next level's
// (the C points' variables, in order)
void variables_init(int n, int nv, DevArray<int>& vars);
void variables_coarsen(int n, const int* states_dev, DevArray<int>& vars);
// keep_states: the states are already set (HMIS / Falgout after the
// Ruge-Stuben passes); otherwise set_initial_states first.
void split_pmis(const rb_csr_s& S, const double* weights_dev, int* states_dev,
                bool keep_states = false);
void split_cljp(const rb_csr_s& S, const double* weights_dev, int* states_dev,
                bool keep_states = false);
// Ruge-Stuben first pass (and second pass) on the host (coarsen_rs.cu).
void split_rs(const rb_csr_s& S, int* states_dev, bool second_pass);
rb_csr_s* interpolation(const rb_csr_s& A, const rb_csr_s& S, const int* states_dev, int kind,
                        double filter, const int* vars = nullptr);
rb_csr_s* spgemm(const rb_csr_s& A, const rb_csr_s& B);
rb_csr_s* rap(const rb_csr_s& A, const rb_csr_s& P, const rb_csr_s* R_in, bool diag_first);
int colour_rows(const rb_csr_s& A, int* colour_dev);

// Smoothed-aggregation setup components (aggregation.cu).  states, agg, r, B
// and R are device arrays.
void mis2(const rb_csr_s& S, const double* r_dev, int* states_dev);
int aggregate(const rb_csr_s& A, const rb_csr_s& S, const int* states_dev, int* agg_dev,
              const double* r_dev);
rb_csr_s* fit_candidates(int n, int n_aggs, const int* agg_dev, const double* B_dev,
                         double* R_dev);
rb_csr_s* jacobi_prolongation(const rb_csr_s& A, const rb_csr_s& T, double omega, int steps);

// Batches of independent systems (batch.cu).
rb_batch_s* batch_setup(int n, const rb_csr_s* const* mats, const rb_amg_opts& o);
void batch_destroy(rb_batch_s* B);
int batch_num_systems(const rb_batch_s* B);
long long batch_offset(const rb_batch_s* B, int s);
int batch_levels(const rb_batch_s* B, int s);
int batch_packed_levels(const rb_batch_s* B);
void batch_cycle(rb_batch_s* B, double* x, const double* b);
int batch_host_waits(const rb_batch_s* B);
int batch_pcg(rb_batch_s* B, double* x, const double* b, double tol, int max_iter, int* iters,
              double* relres);

// Differentiation form (adjoint.cu).
rb_csr_s* fv_assemble(int nx, int ny, const double* k_dev);
void fv_backward(int nx, int ny, const double* k_dev, const rb_csr_s& A, const double* gA,
                 double* gk);
void sddmm(const rb_csr_s& A, const double* lambda, const double* x, double scale, double* out);
bool is_symmetric(const rb_csr_s& A, double tol);

// glibc rand() weights of the reference (par_multilevel.hpp:215-225).
std::vector<double> rand_weights(int n, int first_row);

}  // namespace rb
