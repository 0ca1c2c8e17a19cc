/* raptor_b200.hpp -- header-only C++ shim over the C ABI that re-exposes the
 * reference's AMG solve path (13manan/raptor) at world size 1 with its class
 * and function names, so a caller of the reference changes the include and
 * keeps its code:
 *
 *   ParCSRMatrix* A = par_stencil_grid(stencil, grid, 3);   (gallery/par_stencil.hpp:16)
 *   ParVector x(n, n), b(n, n);                             (core/par_vector.hpp:60)
 *   A->mult(x, b); A->residual(x, b, r);                    (core/par_matrix.hpp:243-250)
 *   ParMultilevel* ml = new ParRugeStubenSolver(0.25, PMIS, Extended, Classical, SOR);
 *   ml->relax_weight = ...; ml->setup(A); ml->solve(x, b);   (multilevel/par_multilevel.hpp)
 *   PCG(A, ml, x, b, res, 1e-8);                            (krylov/par_cg.hpp:14)
 *   Pre_BiCGStab(A, x, b, ml, res, 1e-8);                   (krylov/par_bicgstab.hpp:15)
 *
 * Everything lives in namespace raptor_b200 (pull it in with a using
 * declaration where the reference code says `using namespace raptor`).
 * Errors throw raptor_b200::error carrying the C status code and message (the
 * reference prints and exits).  Objects own their device memory; copies are
 * disabled. */
#ifndef RAPTOR_B200_HPP
#define RAPTOR_B200_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "raptor_b200.h"

namespace raptor_b200 {

template <typename T>
using aligned_vector = std::vector<T>;

enum coarsen_t { RS, CLJP, Falgout, PMIS, HMIS };           /* core/types.hpp:160 */
enum interp_t { Direct, ModClassical, Extended };           /* core/types.hpp:161 */
enum strength_t { Classical, Symmetric };                   /* core/types.hpp:158 */
enum relax_t { Jacobi, SOR, SSOR, L1Jacobi };               /* core/types.hpp:164 (+ L1Jacobi) */
enum agg_t { MIS };                                         /* core/types.hpp:162 */
enum prolong_t { JacobiProlongation };                      /* core/types.hpp:163 */

struct error : std::runtime_error {
    int code;
    error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != RB_OK) throw error(rc, std::string("raptor_b200: ") + rb_last_error());
}

class ParVector {
  public:
    ParVector(int global_n, int local_n) : n_(local_n) {
        (void)global_n;
        check(rb_vec_create(local_n, &h_));
    }
    explicit ParVector(int n) : ParVector(n, n) {}
    ParVector(const ParVector&) = delete;
    ParVector& operator=(const ParVector&) = delete;
    ~ParVector() { rb_vec_destroy(h_); }

    int size() const { return n_; }
    rb_vec handle() const { return h_; }
    void set_const_value(double v) { check(rb_vec_set(h_, v)); }
    void set_values(const double* host_or_device) { check(rb_vec_upload(h_, host_or_device)); }
    void get_values(double* host_or_device) const { check(rb_vec_download(h_, host_or_device)); }
    void copy(const ParVector& y) { check(rb_vec_copy(h_, y.h_)); }
    void axpy(const ParVector& x, double alpha) { check(rb_vec_axpy(h_, x.h_, alpha)); }
    void scale(double alpha) { check(rb_vec_scale(h_, alpha)); }
    double inner_product(const ParVector& x) const {
        double d = 0;
        check(rb_vec_dot(h_, x.h_, &d));
        return d;
    }
    double norm(int p) const {
        if (p != 2) throw error(RB_ERR_INVALID, "raptor_b200: only the 2-norm is provided");
        double d = 0;
        check(rb_vec_norm2(h_, &d));
        return d;
    }

  private:
    rb_vec h_ = nullptr;
    int n_ = 0;
};

class ParCSRMatrix {
  public:
    explicit ParCSRMatrix(rb_csr h) : h_(h) {
        int64_t z = 0;
        check(rb_csr_info(h_, &global_num_rows, &global_num_cols, &z));
        local_num_rows = global_num_rows;
        local_nnz = (long)z;
    }
    /* host CSR arrays (copied to the device) */
    ParCSRMatrix(int n_rows, int n_cols, const int* rowptr, const int* cols, const double* vals) {
        check(rb_csr_create(n_rows, n_cols, rowptr[n_rows], rowptr, cols, vals, 0, &h_));
        global_num_rows = local_num_rows = n_rows;
        global_num_cols = n_cols;
        local_nnz = rowptr[n_rows];
    }
    ParCSRMatrix(const ParCSRMatrix&) = delete;
    ParCSRMatrix& operator=(const ParCSRMatrix&) = delete;
    ~ParCSRMatrix() { rb_csr_destroy(h_); }

    rb_csr handle() const { return h_; }
    void mult(ParVector& x, ParVector& b) { check(rb_spmv(h_, x.handle(), b.handle())); }
    void residual(ParVector& x, ParVector& b, ParVector& r) {
        check(rb_residual(h_, x.handle(), b.handle(), r.handle()));
    }
    void mult_T(ParVector& x, ParVector& b) { check(rb_spmv_T(h_, x.handle(), b.handle())); }
    void mult_append(ParVector& x, ParVector& b) {
        check(rb_spmv_append(h_, x.handle(), b.handle()));
    }
    ParCSRMatrix* mult(ParCSRMatrix* B) {
        rb_csr C = nullptr;
        check(rb_spgemm(h_, B->h_, &C));
        return new ParCSRMatrix(C);
    }

    int global_num_rows = 0, global_num_cols = 0, local_num_rows = 0;
    long local_nnz = 0;

  private:
    rb_csr h_ = nullptr;
};

/* gallery/diffusion.hpp:58 -- new[]'d 9-point stencil, caller deletes */
inline double* diffusion_stencil_2d(double eps = 1.0, double theta = 0.0) {
    double* s = new double[9];
    check(rb_diffusion_stencil_2d(eps, theta, s));
    return s;
}
/* gallery/laplacian27pt.hpp:27 -- new[]'d 27-point stencil */
inline double* laplace_stencil_27pt() {
    double* s = new double[27];
    check(rb_laplace_stencil_27pt(s));
    return s;
}
/* gallery/par_stencil.hpp:16 */
inline ParCSRMatrix* par_stencil_grid(const double* stencil, const int* grid, int dim) {
    rb_csr h = nullptr;
    check(rb_stencil_grid(stencil, grid, dim, &h));
    return new ParCSRMatrix(h);
}
/* gallery/par_matrix_IO.hpp:20 (PETSc binary) */
inline ParCSRMatrix* readParMatrix(const char* filename) {
    rb_csr h = nullptr;
    check(rb_read_petsc(filename, &h));
    return new ParCSRMatrix(h);
}
/* gallery/matrix_market.hpp, gallery/par_matrix_market.hpp (MatrixMarket
 * coordinate files; see rb_read_mm / rb_read_par_mm for the two readers'
 * conventions) */
inline ParCSRMatrix* read_mm(const char* fname) {
    rb_csr h = nullptr;
    check(rb_read_mm(fname, &h));
    return new ParCSRMatrix(h);
}
inline ParCSRMatrix* read_par_mm(const char* fname) {
    rb_csr h = nullptr;
    check(rb_read_par_mm(fname, &h));
    return new ParCSRMatrix(h);
}
inline void write_mm(ParCSRMatrix* A, const char* fname) { check(rb_write_mm(A->handle(), fname)); }
inline void write_par_mm(ParCSRMatrix* A, const char* fname) { write_mm(A, fname); }

/* multilevel/par_multilevel.hpp: the option fields are the C options
 * themselves, so `ml->relax_weight = w` and friends work as in the reference */
/* BSRMatrix (core/matrix.hpp:962-1060): n_rows x n_cols blocks of b_rows x
 * b_cols values; block j's values at vals[j*b_rows*b_cols], row-major. */
class BSRMatrix {
  public:
    explicit BSRMatrix(rb_bsr h) : h_(h) {
        int64_t z = 0;
        check(rb_bsr_info(h_, &n_rows, &n_cols, &b_rows, &b_cols, &z));
        nnz = (long)z;
    }
    /* host block CSR arrays (copied to the device) */
    BSRMatrix(int num_block_rows, int num_block_cols, int block_row_size, int block_col_size,
              const int* rowptr, const int* cols, const double* vals) {
        check(rb_bsr_create(num_block_rows, num_block_cols, block_row_size, block_col_size,
                            rowptr[num_block_rows], rowptr, cols, vals, 0, &h_));
        n_rows = num_block_rows;
        n_cols = num_block_cols;
        b_rows = block_row_size;
        b_cols = block_col_size;
        nnz = rowptr[num_block_rows];
    }
    BSRMatrix(const BSRMatrix&) = delete;
    BSRMatrix& operator=(const BSRMatrix&) = delete;
    ~BSRMatrix() { rb_bsr_destroy(h_); }

    rb_bsr handle() const { return h_; }
    void mult(ParVector& x, ParVector& b) { check(rb_bsr_spmv(h_, x.handle(), b.handle())); }
    void mult_T(ParVector& x, ParVector& b) { check(rb_bsr_spmv_T(h_, x.handle(), b.handle())); }
    void mult_append(ParVector& x, ParVector& b) {
        check(rb_bsr_spmv_append(h_, x.handle(), b.handle()));
    }
    void residual(ParVector& x, ParVector& b, ParVector& r) {
        check(rb_bsr_residual(h_, x.handle(), b.handle(), r.handle()));
    }
    /* BSRMatrix::to_CSR (core/matrix.cpp:1180-1185); the caller owns it */
    ParCSRMatrix* to_CSR() {
        rb_csr C = nullptr;
        check(rb_bsr_to_csr(h_, &C));
        return new ParCSRMatrix(C);
    }

    int n_rows = 0, n_cols = 0, b_rows = 1, b_cols = 1;
    long nnz = 0;

  private:
    rb_bsr h_ = nullptr;
};

class ParMultilevel {
  public:
    virtual ~ParMultilevel() {
        if (h_) rb_amg_destroy(h_);
    }
    ParMultilevel(const ParMultilevel&) = delete;
    ParMultilevel& operator=(const ParMultilevel&) = delete;

    void setup(ParCSRMatrix* Af) {
        if (h_) rb_amg_destroy(h_);
        h_ = nullptr;
        check(rb_amg_setup(Af->handle(), &opts, nullptr, &h_));
        int nl = 0;
        check(rb_amg_num_levels(h_, &nl));
        num_levels = nl;
    }
    int solve(ParVector& sol, ParVector& rhs) {
        residuals.assign((size_t)opts.max_iterations + 1, 0.0);
        int iters = 0;
        const int rc = rb_amg_solve(h_, sol.handle(), rhs.handle(), &iters, residuals.data(),
                                    (int)residuals.size());
        if (rc != RB_OK && rc != RB_ERR_NOT_CONVERGED) check(rc);
        residuals.resize((size_t)iters + 1);
        return iters;
    }
    void cycle(ParVector& x, ParVector& b) { check(rb_amg_cycle(h_, x.handle(), b.handle())); }
    aligned_vector<double>& get_residuals() { return residuals; }
    rb_amg handle() const { return h_; }

    rb_amg_opts opts;
    int& num_smooth_sweeps = opts.num_smooth_sweeps;
    int& max_coarse = opts.max_coarse;
    int& max_levels = opts.max_levels;
    int& max_iterations = opts.max_iterations;
    double& strong_threshold = opts.strong_threshold;
    double& relax_weight = opts.relax_weight;
    double& solve_tol = opts.solve_tol;
    int& precision = opts.precision;
    int num_levels = 0;

  protected:
    ParMultilevel(double theta, strength_t strength, relax_t relax) {
        rb_amg_default_opts(&opts);
        opts.strong_threshold = theta;
        opts.strength_type = strength;
        opts.relax_type = relax;
    }
    rb_amg h_ = nullptr;
    aligned_vector<double> residuals;
};

/* ruge_stuben/par_ruge_stuben_solver.hpp:24 */
class ParRugeStubenSolver : public ParMultilevel {
  public:
    ParRugeStubenSolver(double strong_threshold = 0.0, coarsen_t coarsen_type = RS,
                        interp_t interp_type = Direct, strength_t strength_type = Classical,
                        relax_t relax_type = SOR)
        : ParMultilevel(strong_threshold, strength_type, relax_type) {
        if (interp_type != Direct && interp_type != ModClassical && interp_type != Extended)
            throw error(RB_ERR_INVALID, "raptor_b200: interpolation is Direct, ModClassical or Extended");
        opts.solver = RB_SOLVER_RS;
        opts.coarsen_type = (int)coarsen_type;
        opts.interp_type = interp_type;
    }
    double& interp_filter = opts.interp_filter;
    int& num_variables = opts.num_variables;   /* ParMultilevel::num_variables */
};

/* aggregation/par_smoothed_aggregation_solver.hpp:17 */
class ParSmoothedAggregationSolver : public ParMultilevel {
  public:
    ParSmoothedAggregationSolver(double strong_threshold = 0.0, agg_t agg_type = MIS,
                                 prolong_t prolong_type = JacobiProlongation,
                                 strength_t strength_type = Symmetric, relax_t relax_type = SOR,
                                 int prolong_smooth_steps = 1, double prolong_weight = 4.0 / 3)
        : ParMultilevel(strong_threshold, strength_type, relax_type) {
        (void)agg_type;
        (void)prolong_type;
        opts.solver = RB_SOLVER_SA;
        opts.prolong_smooth_steps = prolong_smooth_steps;
        opts.prolong_weight = prolong_weight;
    }
};

namespace detail {
inline int hist_cap(const ParCSRMatrix* A, int max_iter) {
    return (max_iter > 0 ? max_iter : (int)(1.3 * A->global_num_rows) + 2) + 2;
}
}  // namespace detail

/* krylov/par_cg.hpp:14 -- the reference's stopping rule and history */
inline void PCG(ParCSRMatrix* A, ParMultilevel* ml, ParVector& x, ParVector& b,
                aligned_vector<double>& res, double tol = 1e-05, int max_iter = -1) {
    res.assign((size_t)detail::hist_cap(A, max_iter), 0.0);
    int nh = 0;
    const int rc = rb_pcg(A->handle(), ml->handle(), x.handle(), b.handle(), tol, max_iter,
                          RB_PCG_REFERENCE, res.data(), (int)res.size(), &nh);
    if (rc != RB_OK && rc != RB_ERR_NOT_CONVERGED) check(rc);
    res.resize((size_t)nh);
}
/* krylov/par_cg.hpp:12 */
inline void CG(ParCSRMatrix* A, ParVector& x, ParVector& b, aligned_vector<double>& res,
               double tol = 1e-05, int max_iter = -1) {
    res.assign((size_t)detail::hist_cap(A, max_iter), 0.0);
    int nh = 0;
    const int rc = rb_cg(A->handle(), x.handle(), b.handle(), tol, max_iter, res.data(),
                         (int)res.size(), &nh);
    if (rc != RB_OK && rc != RB_ERR_NOT_CONVERGED) check(rc);
    res.resize((size_t)nh);
}
/* krylov/par_bicgstab.hpp:13 */
inline void BiCGStab(ParCSRMatrix* A, ParVector& x, ParVector& b, aligned_vector<double>& res,
                     double tol = 1e-05, int max_iter = -1) {
    res.assign((size_t)detail::hist_cap(A, max_iter), 0.0);
    int nh = 0;
    const int rc = rb_bicgstab(A->handle(), nullptr, x.handle(), b.handle(), tol, max_iter,
                               res.data(), (int)res.size(), &nh);
    if (rc != RB_OK && rc != RB_ERR_NOT_CONVERGED) check(rc);
    res.resize((size_t)nh);
}
/* krylov/par_bicgstab.hpp:15 */
inline void Pre_BiCGStab(ParCSRMatrix* A, ParVector& x, ParVector& b, ParMultilevel* ml,
                         aligned_vector<double>& res, double tol = 1e-05, int max_iter = -1) {
    res.assign((size_t)detail::hist_cap(A, max_iter), 0.0);
    int nh = 0;
    const int rc = rb_bicgstab(A->handle(), ml->handle(), x.handle(), b.handle(), tol, max_iter,
                               res.data(), (int)res.size(), &nh);
    if (rc != RB_OK && rc != RB_ERR_NOT_CONVERGED) check(rc);
    res.resize((size_t)nh);
}

}  // namespace raptor_b200

#endif /* RAPTOR_B200_HPP */
