/*
 * raptor_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement, in plain C99, of RAPtor's AMG path at MPI world size 1
 * (13manan/raptor).  It is the checker that the CUDA product is compared
 * against: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference leg load it.  Nothing in the product links or calls it.
 *
 * Every function restates the reference loop it cites (file:line within the
 * reference project), including the reference's quirks:
 *   - the parallel Jacobi smoother never updates x (par_relax.cpp:127,146);
 *     `jacobi_compat=1` reproduces that, `jacobi_compat=0` is weighted Jacobi;
 *   - forward SOR uses x=(x+w(b-x-sum))/d (par_relax.cpp:66);
 *   - SpGEMM emits rows in reverse insertion order and drops |s|<=1e-16
 *     (util/linalg/matmult.cpp:71-137), then add_append sorts and drops
 *     |v|<1e-16 (util/linalg/add.cpp:39-78, core/matrix.cpp remove_duplicates);
 *   - the coarse LU factors A_c^T (row-major dense into column-major dgetrf,
 *     multilevel/par_multilevel.hpp:229-339, :365-374);
 *   - PCG stops on r.z < tol*sqrt(b.Mb) and restarts every 8 iterations
 *     (krylov/par_cg.cpp:121-263).
 * Parity of this restatement is pinned against the reference's own golden
 * fixtures (test_data/*.pm, *.txt) by tests/test_oracle_golden.py, and against
 * the reference's sequential sources compiled under oracle/_ref.
 */
#ifndef RAPTOR_ORACLE_H
#define RAPTOR_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oc_csr {
    int n_rows, n_cols, nnz, cap;
    int* rowptr;
    int* cols;
    double* vals;
} oc_csr;

/* state codes, core/types.hpp:31-37 */
#define OC_SELECTED 1
#define OC_UNSELECTED 0
#define OC_UNASSIGNED -1
#define OC_NONEIGHBORS -2
#define OC_NEWSELECTION 3
#define OC_NEWUNSELECTION 2

/* relaxation kinds (the first three are core/types.hpp:164 relax_t) */
#define OC_RELAX_JACOBI 0
#define OC_RELAX_SOR 1
#define OC_RELAX_SSOR 2
#define OC_RELAX_L1JACOBI 3
#define OC_RELAX_MCSOR 4
#define OC_RELAX_MCSSOR 5

/* setup kinds */
#define OC_INTERP_DIRECT 0
#define OC_INTERP_MODCLASSICAL 1
#define OC_INTERP_EXTENDED 2
#define OC_SOLVER_RS 0
#define OC_SOLVER_SA 1

typedef struct oc_opts {
    int solver;            /* OC_SOLVER_RS / OC_SOLVER_SA */
    int interp;            /* RS: OC_INTERP_* */
    int relax;             /* OC_RELAX_* */
    int jacobi_compat;     /* 1: reference jacobi_helper (x untouched) */
    int num_smooth_sweeps; /* par_multilevel.hpp:87 */
    int max_coarse;        /* :89 */
    int max_levels;        /* :90 */
    int max_iterations;    /* :99 */
    double strong_threshold;
    double relax_weight;   /* :88 */
    double solve_tol;      /* :98 */
    double interp_filter;  /* par_ruge_stuben_solver.hpp:24 */
    double prolong_weight; /* par_smoothed_aggregation_solver.hpp:23 */
    int prolong_smooth_steps;
    int seed_offset;       /* first_local_row added to 2448422 (0 at WS1) */
} oc_opts;

typedef struct oc_level {
    oc_csr* A;
    oc_csr* P;
    int n;
    double* x;
    double* b;
    double* tmp;
    int* colour;      /* multicolour smoothers: colour of each row */
    int n_colours;
    double* l1;       /* L1-Jacobi row norms */
} oc_level;

typedef struct oc_ml {
    oc_opts o;
    int num_levels;
    oc_level lv[40];
    int coarse_n;
    double* lu;       /* column-major LU of A_c^T (dgetrf semantics) */
    int* piv;
} oc_ml;

/* containers */
oc_csr* oc_csr_new(int n_rows, int n_cols, int nnz, const int* rowptr,
                   const int* cols, const double* vals);
oc_csr* oc_csr_copy(const oc_csr* A);
void oc_csr_free(oc_csr* A);
void oc_csr_info(const oc_csr* A, int* n_rows, int* n_cols, int* nnz);
void oc_csr_export(const oc_csr* A, int* rowptr, int* cols, double* vals);
void oc_csr_sort(oc_csr* A);
void oc_csr_move_diag(oc_csr* A);
oc_csr* oc_csr_transpose(const oc_csr* A);

/* gallery: gallery/par_stencil.hpp, diffusion.hpp, laplacian27pt.hpp */
void oc_diffusion_stencil_2d(double eps, double theta, double* out9);
void oc_laplace_stencil_27pt(double* out27);
oc_csr* oc_stencil_grid(const double* stencil, const int* grid, int dim);

/* SpMV family: util/linalg/spmv.cpp */
/* Threads for the row-parallel loops (SpMV, residual, append, Jacobi and
 * L1-Jacobi sweeps, axpy): each row is still computed alone and in the same
 * order, so results do not depend on the count; dots and the transposed
 * (scatter) product stay sequential.  Default 1.  Used by the CPU baseline
 * timing; only effective when built with OpenMP. */
void oc_set_threads(int n);
int oc_get_threads(void);
void oc_spmv(const oc_csr* A, const double* x, double* b);
void oc_residual(const oc_csr* A, const double* x, const double* b, double* r);
void oc_spmv_T(const oc_csr* A, const double* x, double* b);
void oc_spmv_append(const oc_csr* A, const double* x, double* b);

/* block CSR: nbr x nbc blocks of br x bc values, block j's values at
 * vals[j*br*bc], row-major (core/matrix.hpp:962-1060, util/linalg/spmv.cpp) */
void oc_bsr_spmv(int nbr, int br, int bc, const int* rowptr, const int* cols,
                 const double* vals, const double* x, double* b);
void oc_bsr_append(int nbr, int br, int bc, const int* rowptr, const int* cols,
                   const double* vals, const double* x, double* b);
void oc_bsr_residual(int nbr, int br, int bc, const int* rowptr, const int* cols,
                     const double* vals, const double* x, const double* b, double* r);
void oc_bsr_spmv_T(int nbr, int nbc, int br, int bc, const int* rowptr, const int* cols,
                   const double* vals, const double* x, double* b);
oc_csr* oc_bsr_to_csr(int nbr, int nbc, int br, int bc, const int* rowptr, const int* cols,
                      const double* vals);

/* setup components */
oc_csr* oc_classical_strength(const oc_csr* A, double theta);
oc_csr* oc_symmetric_strength(const oc_csr* A, double theta);
void oc_split_pmis(const oc_csr* S, const double* rand_vals, int* states);
void oc_split_cljp(const oc_csr* S, const double* rand_vals, int* states);
void oc_split_rs(const oc_csr* S, int* states, int prev_states, int second_pass);
oc_csr* oc_mod_classical_interp(const oc_csr* A, const oc_csr* S, const int* states);
oc_csr* oc_direct_interp(const oc_csr* A, const oc_csr* S, const int* states);
oc_csr* oc_extended_interp(const oc_csr* A, const oc_csr* S, const int* states,
                           double filter);
oc_csr* oc_spgemm(const oc_csr* A, const oc_csr* B);
oc_csr* oc_spgemm_T(const oc_csr* P, const oc_csr* B);
oc_csr* oc_rap(const oc_csr* A, const oc_csr* P, int sort_diag_first);
void oc_mis2(const oc_csr* S, const double* rand_vals, int* states);
int oc_aggregate(const oc_csr* A, const oc_csr* S, int* states, int* aggregates,
                 const double* r);
oc_csr* oc_fit_candidates(int n, int n_aggs, const int* aggregates,
                          const double* B, double* R, double tol);
oc_csr* oc_jacobi_prolongation(const oc_csr* A, const oc_csr* T, double omega,
                               int steps);
int oc_colour_rows(const oc_csr* A, int* colour);

/* hierarchy + solve path */
void oc_default_opts(oc_opts* o);
oc_ml* oc_ml_setup(const oc_csr* A, const oc_opts* o, const double* weights,
                   int n_weights);
void oc_ml_free(oc_ml* ml);
int oc_ml_num_levels(const oc_ml* ml);
const oc_csr* oc_ml_level_A(const oc_ml* ml, int l);
const oc_csr* oc_ml_level_P(const oc_ml* ml, int l);
void oc_ml_cycle(oc_ml* ml, double* x, const double* b);
int oc_ml_solve(oc_ml* ml, double* x, const double* b, double* hist, int cap);
int oc_pcg(const oc_csr* A, oc_ml* ml, double* x, const double* b, double tol,
           int max_iter, double* hist, int cap);
int oc_pcg_mode(const oc_csr* A, oc_ml* ml, double* x, const double* b, double tol,
                int max_iter, int mode, double* hist, int cap);
int oc_cg(const oc_csr* A, double* x, const double* b, double tol, int max_iter,
          double* hist, int cap);
int oc_bicgstab(const oc_csr* A, double* x, const double* b, double tol,
                int max_iter, double* hist, int cap);
int oc_pre_bicgstab(const oc_csr* A, oc_ml* ml, double* x, const double* b,
                    double tol, int max_iter, double* hist, int cap);
void oc_form_rand_weights(int n, int first_row, double* w);
void oc_dense_lu(int n, double* a_colmajor, int* piv);
void oc_dense_lu_solve(int n, const double* lu, const int* piv, double* b);

#ifdef __cplusplus
}
#endif
#endif
