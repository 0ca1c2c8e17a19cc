/*
 * raptor_b200.h -- C ABI of libraptor_b200, a B200-native (sm_100a) rebuild
 * of RAPtor's algebraic-multigrid solve path at MPI world size 1.
 *
 * Plain C: opaque handles, pointers and sizes, integer status codes.  Every
 * call is ordered on the library stream (rb_set_stream) and returns RB_OK or a
 * negative rb_status; rb_last_error() describes the last failure of the
 * calling thread.  One handle is used by one host thread at a time.
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the reference project 13manan/raptor).  At world size 1 a ParCSRMatrix is
 * its on_proc block, so one device CSR matrix stands for it.
 */
#ifndef RAPTOR_B200_H
#define RAPTOR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------- status */
typedef enum rb_status {
    RB_OK = 0,
    RB_ERR_INVALID = -1,       /* bad argument or size mismatch (par_vector.cpp:105-111 exits) */
    RB_ERR_CUDA = -2,          /* CUDA runtime failure */
    RB_ERR_OOM = -3,           /* device allocation failed */
    RB_ERR_BREAKDOWN = -4,     /* p.Ap < 0 in CG (par_cg.cpp:195-202 exits) or NaN in a dot */
    RB_ERR_NOT_CONVERGED = -5, /* iteration limit reached without meeting the tolerance */
    RB_ERR_NO_DEVICE = -6      /* no CUDA device or the kernels are missing for it */
} rb_status;

typedef struct rb_csr_s* rb_csr;   /* device CSR matrix, FP64 values, int32 indices */
typedef struct rb_vec_s* rb_vec;   /* device FP64 vector */
typedef struct rb_amg_s* rb_amg;   /* AMG hierarchy (ParMultilevel) */
typedef struct rb_batch_s* rb_batch; /* independent systems solved together */
typedef struct rb_bsr_s* rb_bsr;   /* device block CSR matrix, FP64 blocks, int32 block indices */

/* Description of the last failure on this thread ("" when none). */
const char* rb_last_error(void);
/* Select the CUDA device and create the library stream. */
int rb_init(int device);
/* Order all later calls on a caller-owned stream (0 = library stream). */
int rb_set_stream(void* cuda_stream);
/* Wait for all work queued on the library stream. */
int rb_synchronize(void);
/* Library version string. */
const char* rb_version(void);

/* ------------------------------------------------------------ containers */
/* ParCSRMatrix(...) + finalize (core/par_matrix.hpp:481-611, par_matrix.cpp:111-157).
 * Copies host (on_device=0) or device (on_device=1) arrays. */
int rb_csr_create(int n_rows, int n_cols, int64_t nnz, const int* rowptr, const int* cols,
                  const double* vals, int on_device, rb_csr* out);
int rb_csr_destroy(rb_csr A);
int rb_csr_info(rb_csr A, int* n_rows, int* n_cols, int64_t* nnz);
/* Copy the matrix to host buffers of n_rows+1, nnz and nnz entries. */
int rb_csr_download(rb_csr A, int* rowptr, int* cols, double* vals);
/* Device pointers of the matrix arrays (borrowed).  Values may be rewritten
 * in place between calls; the pattern (rowptr, cols) may not. */
int rb_csr_device_arrays(rb_csr A, int** rowptr, int** cols, double** vals);
/* CSRMatrix::sort then move_diag (core/matrix.cpp:588-618, :730-786). */
int rb_csr_sort_diag_first(rb_csr A);
/* Transpose with rows of the result in increasing source-row order
 * (CSRMatrix::transpose / CSR_to_CSC, core/matrix.cpp:148-154, :492-538). */
int rb_csr_transpose(rb_csr A, rb_csr* out);

/* Block CSR (BSRMatrix, core/matrix.hpp:962-1060): n_block_rows x
 * n_block_cols blocks of b_rows x b_cols values; rowptr (n_block_rows+1) and
 * cols (nnz_blocks) index blocks, and block j's values are
 * vals[j*b_rows*b_cols ...], row-major inside the block (the reference's
 * block_vals[j][r*b_cols + c]).  Copies host (on_device=0, checked) or device
 * (on_device=1) arrays.  Vectors of a product hold scalar entries:
 * n_block_cols*b_cols for x, n_block_rows*b_rows for b. */
int rb_bsr_create(int n_block_rows, int n_block_cols, int b_rows, int b_cols, int64_t nnz_blocks,
                  const int* rowptr, const int* cols, const double* vals, int on_device,
                  rb_bsr* out);
int rb_bsr_destroy(rb_bsr A);
int rb_bsr_info(rb_bsr A, int* n_block_rows, int* n_block_cols, int* b_rows, int* b_cols,
                int64_t* nnz_blocks);
/* Copy the matrix to host buffers of n_block_rows+1, nnz_blocks and
 * nnz_blocks*b_rows*b_cols entries (a NULL buffer is skipped). */
int rb_bsr_download(rb_bsr A, int* rowptr, int* cols, double* vals);
/* b = A x: BSRMatrix::spmv / BSR_spmv (util/linalg/spmv.cpp:121-148, 343-346). */
int rb_bsr_spmv(rb_bsr A, rb_vec x, rb_vec b);
/* b += A x: BSRMatrix::spmv_append / BSR_append (spmv.cpp:105-119, 347-350). */
int rb_bsr_spmv_append(rb_bsr A, rb_vec x, rb_vec b);
/* r = b - A x: BSRMatrix::spmv_residual (spmv.cpp:363-368). */
int rb_bsr_residual(rb_bsr A, rb_vec x, rb_vec b, rb_vec r);
/* b = A^T x: Matrix::mult_T with the block append_T (core/matrix.hpp:342-348,
 * 299-312).  The first call builds the transposed block pattern on the
 * handle (host counting sort, then kept); later calls allocate nothing. */
int rb_bsr_spmv_T(rb_bsr A, rb_vec x, rb_vec b);
/* Scalar CSR of the matrix, entries with |v| > 1e-16 in the reference's
 * order: BSRMatrix::to_CSR / BSR_to_CSR (core/matrix.cpp:1180-1185, 358-395). */
int rb_bsr_to_csr(rb_bsr A, rb_csr* out);

/* ParVector (core/par_vector.hpp:44-176) */
int rb_vec_create(int n, rb_vec* out);
int rb_vec_destroy(rb_vec v);
int rb_vec_size(rb_vec v, int* n);
int rb_vec_upload(rb_vec v, const double* host);   /* host or device source */
int rb_vec_download(rb_vec v, double* host);       /* host or device destination */
int rb_vec_set(rb_vec v, double value);          /* ParVector::set_const_value */
int rb_vec_device_ptr(rb_vec v, double** ptr);
int rb_vec_copy(rb_vec dst, rb_vec src);         /* ParVector::copy */
int rb_vec_axpy(rb_vec y, rb_vec x, double a);   /* ParVector::axpy, vector.cpp:53-59 */
int rb_vec_scale(rb_vec y, double a);            /* ParVector::scale, vector.cpp:89-95 */
/* out[k] = x[idx[k]] for k < n, idx and out device pointers (ordered on the
 * library stream): the send-buffer packing of a halo exchange, ParComm's
 * init_comm / pack_values (core/comm_pkg.hpp:145-158, core/comm_data.hpp:
 * 257-262, 584).  An index outside x writes NaN. */
int rb_vec_gather(rb_vec x, const int* idx, int n, double* out);
/* y[idx[k]] += vals[k] for k < n, idx and vals device pointers: adding the
 * values a transpose halo exchange receives into the owner's rows, ParComm's
 * complete_comm_T (core/comm_pkg.hpp:198-211).  The indices of one call must
 * be distinct (call once per message); an index outside y is skipped. */
int rb_vec_scatter_add(rb_vec y, const int* idx, const double* vals, int n);
int rb_vec_dot(rb_vec a, rb_vec b, double* out); /* ParVector::inner_product, par_vector.cpp:101-121 */
int rb_vec_norm2(rb_vec a, double* out);         /* ParVector::norm(2), par_vector.cpp:88-98 */

/* --------------------------------------------------------- SpMV family */
/* ParMatrix::mult, b = A x (util/linalg/par_spmv.cpp:25-59 -> spmv.cpp:52-67).
 * The first product (of rb_spmv, rb_residual or rb_spmv_append) on a matrix
 * times the row schedules once and keeps the fastest on the handle. */
int rb_spmv(rb_csr A, rb_vec x, rb_vec b);
/* ParMatrix::residual, r = b - A x (par_spmv.cpp:215-252 -> spmv.cpp:69-85) */
int rb_residual(rb_csr A, rb_vec x, rb_vec b, rb_vec r);
/* ParMatrix::mult_T, b = A^T x (par_spmv.cpp:157-187 -> spmv.cpp:150-163).
 * The first call on a matrix builds and keeps A^T's pattern on the handle;
 * later calls gather A's current values through it. */
int rb_spmv_T(rb_csr A, rb_vec x, rb_vec b);
/* ParMatrix::mult_append, b += A x (par_spmv.cpp:91-125 -> spmv.cpp:88-103) */
int rb_spmv_append(rb_csr A, rb_vec x, rb_vec b);

/* --------------------------------------------------------------- gallery */
/* diffusion_stencil_2d (gallery/diffusion.hpp:58-85) */
int rb_diffusion_stencil_2d(double eps, double theta, double* out9);
/* laplace_stencil_27pt (gallery/laplacian27pt.hpp:27-37) */
int rb_laplace_stencil_27pt(double* out27);
/* par_stencil_grid (gallery/par_stencil.hpp:16-236) */
int rb_stencil_grid(const double* stencil, const int* grid, int dim, rb_csr* out);
/* readParMatrix for PETSc binary AIJ files (gallery/par_matrix_IO.cpp:22+):
 * big-endian int32 header (1211216, rows, columns, nonzeros), row lengths,
 * column indices, float64 values; rows sorted diagonal first as finalize()
 * does.  A file whose row lengths do not add up to the nonzero count, or
 * with a column out of range, is refused (RB_ERR_INVALID). */
int rb_read_petsc(const char* path, rb_csr* out);
/* The same parsing into caller-owned host arrays in file order (no device
 * needed; readMatrix, gallery/matrix_IO.cpp:24-110).  Call with rowptr,
 * cols, vals NULL to learn the sizes, then with arrays of n_rows + 1, nnz
 * and nnz entries. */
int rb_petsc_read_host(const char* path, int* n_rows, int* n_cols, int64_t* nnz, int* rowptr,
                       int* cols, double* vals);
/* Write a PETSc binary AIJ file (what PETSc's MatLoad reads) from host CSR
 * arrays, rows and entries in the given order; the reference reads this
 * format but has no writer.  rb_write_petsc writes a device matrix. */
int rb_petsc_write_host(const char* path, int n_rows, int n_cols, int64_t nnz, const int* rowptr,
                        const int* cols, const double* vals);
int rb_write_petsc(rb_csr A, const char* path);
/* MatrixMarket coordinate files (real, integer or pattern; general,
 * symmetric or skew-symmetric).  read_mm (gallery/matrix_market.cpp:18-76):
 * entries in file order within each row, the symmetry field ignored (the
 * stored triangle only).  read_par_mm (gallery/par_matrix_market.cpp:
 * 18-128): the mirror (j, i) of every off-diagonal entry of a symmetric
 * file is stored too (-v for skew-symmetric) and each row is sorted by
 * column; unlike the reference, a diagonal entry is stored once. */
int rb_read_mm(const char* path, rb_csr* out);
int rb_read_par_mm(const char* path, rb_csr* out);
/* write_mm / write_par_mm (gallery/matrix_market.cpp:78-105): coordinate
 * real general, "i j %2.15e" per entry in row order, 1-based. */
int rb_write_mm(rb_csr A, const char* path);
/* The same parsing into caller-owned host arrays (no device needed; no
 * counterpart in the reference).  mirror = 1 and sort_rows = 1 give
 * read_par_mm's matrix, 0 and 0 read_mm's.  Call with rowptr, cols, vals
 * NULL to learn n_rows, n_cols and nnz, then again with arrays of
 * n_rows + 1, nnz and nnz entries. */
int rb_mm_read_host(const char* path, int mirror, int sort_rows, int* n_rows, int* n_cols,
                    int64_t* nnz, int* rowptr, int* cols, double* vals);
/* write_mm from host CSR arrays (no device needed). */
int rb_mm_write_host(const char* path, int n_rows, int n_cols, int64_t nnz, const int* rowptr,
                     const int* cols, const double* vals);

/* ----------------------------------------------------- setup components */
#define RB_STRENGTH_CLASSICAL 0 /* strength_t Classical (core/types.hpp:158) */
#define RB_STRENGTH_SYMMETRIC 1 /* strength_t Symmetric */
#define RB_INTERP_DIRECT 0       /* interp_t Direct (core/types.hpp:161) */
#define RB_INTERP_MODCLASSICAL 1 /* interp_t ModClassical */
#define RB_INTERP_EXTENDED 2     /* interp_t Extended */
#define RB_COARSEN_RS 0          /* coarsen_t RS (core/types.hpp:160) */
#define RB_COARSEN_CLJP 1        /* coarsen_t CLJP */
#define RB_COARSEN_FALGOUT 2     /* coarsen_t Falgout */
#define RB_COARSEN_PMIS 3        /* coarsen_t PMIS */
#define RB_COARSEN_HMIS 4        /* coarsen_t HMIS */

/* ParCSRMatrix::strength (par_strength.cpp:536-546 -> :8-339 / :342-531).
 * A must have its diagonal first (rb_csr_sort_diag_first). */
int rb_strength(rb_csr A, int kind, double theta, rb_csr* S);
/* split_pmis (ruge_stuben/par_cf_splitting.cpp:75-89, 1229-1381); weights has
 * n_rows entries; states (host, n_rows) receive 1 = C, 0 = F, -2 = isolated. */
int rb_split_pmis(rb_csr S, const double* weights, int* states);
/* The C/F splittings at one rank (par_cf_splitting.cpp): split_rs (:7-30,
 * the Ruge-Stuben passes of cf_splitting.cpp:9-328, run on the host),
 * split_cljp (:32-48, 1383-1607), split_falgout (:50-73), split_pmis
 * (:75-89), split_hmis (:91-112), chosen by kind = RB_COARSEN_*.  weights
 * (n_rows, or NULL for the reference's glibc rand() weights) are used by the
 * CLJP and PMIS loops; states (host, n_rows) receive 1 = C, 0 = F, -2 =
 * isolated. */
int rb_split(rb_csr S, int kind, const double* weights, int* states);
/* mod_classical_interpolation (par_interpolation.cpp:991-1451) and
 * extended_interpolation + filter_interp (:280-989, :175-278). */
int rb_interpolation(rb_csr A, rb_csr S, const int* states, int kind, double filter,
                     rb_csr* P);
/* mis2 (aggregation/par_mis.cpp:204-645) on a strength matrix S with its
 * diagonal first; weights as for rb_split_pmis (NULL = the reference's glibc
 * rand() weights); states (host, n_rows) receive 1 = root, 0 = not a root. */
int rb_mis2(rb_csr S, const double* weights, int* states);
/* aggregate (aggregation/par_aggregate.cpp:5-185): A and S with the
 * diagonal first, states from rb_mis2, r the tie-break weights (NULL = 0, as
 * the solver calls it).  aggregates (host, n_rows) receive each row's root
 * row index (-1 = unaggregated); n_aggs the number of roots. */
int rb_aggregate(rb_csr A, rb_csr S, const int* states, const double* r, int* aggregates,
                 int* n_aggs);
/* fit_candidates with one candidate (aggregation/par_candidates.cpp:6-216):
 * T (n_rows x n_aggs, one entry B_i / R_a per aggregated row, columns = the
 * roots in increasing order) and R (host, n_aggs) the aggregate norms. */
int rb_fit_candidates(int n_rows, int n_aggs, const int* aggregates, const double* B, double* R,
                      rb_csr* T);
/* jacobi_prolongation (aggregation/par_prolongation.cpp:7-104):
 * P = (I - omega D_abs^-1 A)^steps T with D_abs the absolute row sums. */
int rb_jacobi_prolongation(rb_csr A, rb_csr T, double omega, int steps, rb_csr* P);
/* C = A B (ParCSRMatrix::mult, par_matmult.cpp:73-107 -> matmult.cpp:71-137 +
 * add.cpp:39-78): rows sorted by column, |c| <= 1e-16 dropped. */
int rb_spgemm(rb_csr A, rb_csr B, rb_csr* C);
/* A_c = P^T (A P) (par_matmult.cpp:141-196, 387-570), then sort + move_diag
 * when diag_first (ruge_stuben/par_ruge_stuben_solver.hpp:139-143). */
int rb_rap(rb_csr A, rb_csr P, int diag_first, rb_csr* Ac);

/* -------------------------------------------------------------- hierarchy */
#define RB_RELAX_JACOBI 0    /* relax_t Jacobi (core/types.hpp:164) */
#define RB_RELAX_SOR 1       /* relax_t SOR: multicolour forward Gauss-Seidel stand-in */
#define RB_RELAX_SSOR 2      /* relax_t SSOR: multicolour forward + backward */
#define RB_RELAX_L1JACOBI 3  /* L1-Jacobi, x += w (b - A x) / sum_j |a_ij| */
#define RB_SOLVER_RS 0       /* ParRugeStubenSolver */
#define RB_SOLVER_SA 1       /* ParSmoothedAggregationSolver */
#define RB_PREC_FP64 0
#define RB_PREC_FP32 1       /* hierarchy values and V-cycle in FP32 */

/* Fields of ParMultilevel (multilevel/par_multilevel.hpp:626-658),
 * ParRugeStubenSolver (ruge_stuben/par_ruge_stuben_solver.hpp:15-25, 164-170)
 * and ParSmoothedAggregationSolver (par_smoothed_aggregation_solver.hpp:17-32),
 * plus the cycle precision and the reference-compatible Jacobi switch. */
typedef struct rb_amg_opts {
    int solver;               /* RB_SOLVER_RS / RB_SOLVER_SA */
    int strength_type;        /* RB_STRENGTH_*; RS default Classical, SA Symmetric */
    int interp_type;          /* RB_INTERP_* (RS) */
    int relax_type;           /* RB_RELAX_* */
    int num_smooth_sweeps;    /* 1 */
    int max_coarse;           /* 50 */
    int max_levels;           /* 25 */
    int max_iterations;       /* 100 (solve) */
    double strong_threshold;  /* 0.25 in the reference's examples */
    double relax_weight;      /* 1.0 */
    double solve_tol;         /* 1e-7 */
    double interp_filter;     /* 0.3 (Extended) */
    double prolong_weight;    /* 4/3 (SA) */
    int prolong_smooth_steps; /* 1 (SA) */
    int precision;            /* RB_PREC_FP64 / RB_PREC_FP32 */
    int jacobi_compat;        /* 1: Jacobi leaves x unchanged, as par_relax.cpp:127,146 does */
    int seed_offset;          /* first_local_row in srand(2448422 + first_local_row) */
    int fuse_coarse;          /* 1 (default): the bottom levels of the cycle run as one launch of one
                                 thread-block cluster, from the start level that times fastest
                                 (none if no start beats separate launches); 0: never;
                                 k >= 2: from level k-1 if that level qualifies */
    int use_graphs;           /* 1: replay cycles / Krylov iterations from CUDA graphs */
    int const_coef;           /* 1 (default): a diagonal-storage level whose diagonals each hold one
                                 value is read as a mask a row plus those values (same results);
                                 0: the stored values */
    int coarsen_type;         /* RB_COARSEN_* (RS solver): PMIS (default), RS, CLJP, Falgout, HMIS
                                 (par_ruge_stuben_solver.hpp:75-104; RS uses Falgout from level 3) */
    int num_variables;        /* 1 (default); k > 1: the unknown-based systems form of the RS solver
                                 (row i is variable i % k; classical strength and ModClassical /
                                 Extended interpolation couple only rows of one variable,
                                 par_strength.cpp:8-339, par_interpolation.cpp:811,918,1308,1390) */
} rb_amg_opts;

void rb_amg_default_opts(rb_amg_opts* opts);
/* ParMultilevel::setup (par_multilevel.hpp:126-212 + extend_hierarchy +
 * duplicate_coarse :229-339).  weights: n_rows values or NULL for the
 * reference's glibc rand() weights. */
int rb_amg_setup(rb_csr A, const rb_amg_opts* opts, const double* weights, rb_amg* out);
int rb_amg_destroy(rb_amg ml);
int rb_amg_num_levels(rb_amg ml, int* num_levels);
/* rows and nonzeros of A_l and P_l (print_hierarchy, par_multilevel.hpp:540-563) */
int rb_amg_level_info(rb_amg ml, int level, int* n_rows, int64_t* nnz_A, int64_t* nnz_P);
/* FP64 copy of A_l (which=0), P_l (1) or R_l = P_l^T (2). */
int rb_amg_level_matrix(rb_amg ml, int level, int which, rb_csr* out);
/* C/F states of level l (host, n_rows). */
int rb_amg_level_states(rb_amg ml, int level, int* states);
/* ParMultilevel::cycle (par_multilevel.hpp:341-457): one V-cycle on x. */
int rb_amg_cycle(rb_amg ml, rb_vec x, rb_vec b);
/* ParMultilevel::solve (par_multilevel.hpp:459-538).  hist receives
 * ||r_k||/||b|| for k = 0..iters (up to cap entries). */
int rb_amg_solve(rb_amg ml, rb_vec x, rb_vec b, int* iters, double* hist, int cap);

/* Time one V-cycle operation by operation (track_times / print_solve_times,
 * par_multilevel.hpp:343-456, 578-619).  ms receives 8 values per level:
 * [pre-smooth, residual, restriction, prolongation, post-smooth, coarse
 * solve, 0, 0] in milliseconds; n_out = 8 * num_levels. */
int rb_amg_cycle_profile(rb_amg ml, double* ms, int cap, int* n_out);
/* Average milliseconds per launch of one cycle operator over reps launches:
 * op 0 residual with A_l, 1 restriction with R_l, 2 prolongation with P_l,
 * 3 Jacobi sweep with A_l, 6 the first sweep from zero fused with the
 * residual, 7 the first sweep alone (all in the cycle precision), 4 the
 * outer FP64 A p fused with p.Ap on the finest level, 5 one whole
 * preconditioner V-cycle z = M r from a zero guess replayed from its CUDA
 * graph (level is ignored). */
int rb_amg_time_operator(rb_amg ml, int level, int op, int reps, double* ms_per_launch);
/* Wall time of the last rb_amg_setup (seconds) and the autotuner's choices
 * for level l: lanes per row of A_l (0 when A_l is stored by diagonals),
 * P_l and R_l (1..32), plus 64 when the operator runs the blocked row
 * schedule (contiguous rows a block) and 128 when it runs the shared-memory
 * schedule (x's window staged per chunk of rows). */
int rb_amg_setup_seconds(rb_amg ml, double* seconds);
int rb_amg_level_lanes(rb_amg ml, int level, int* lanes_A, int* lanes_P, int* lanes_R);
/* Storage of A_l in the cycle: *ndiag = number of stored diagonals when the
 * autotuner picked the sliced-diagonal layout, 0 for CSR. */
int rb_amg_level_storage(rb_amg ml, int level, int* ndiag);
/* 1 when A_l is stored by diagonals with constant coefficients (every
 * nonzero of a diagonal has one value, as in a constant-coefficient stencil):
 * the cycle's kernels then read one 4-byte mask a row (which of the stencil's
 * entries the row has) in place of the row's values, with the same products
 * in the same order.  2 when, in addition, A_l is a 27-, 7-, 9- or 5-point
 * stencil on a box whose rows hold exactly their in-box neighbours: the
 * kernels then stage x in shared memory plane by plane and read no mask
 * (the same products in the same order again), where the autotuner timed
 * that faster.  RAPTOR_B200_CONST_DIA=0 at setup keeps the values;
 * RAPTOR_B200_GRID_DIA=0 keeps the mask, =1 or =2 take the box form untimed
 * with one or two rows in x a thread.  No
 * counterpart in the reference. */
int rb_amg_level_const_coef(rb_amg ml, int level, int* constant);
/* 1 when level l's first sweep from zero runs fused with its residual (one
 * pass over A_l; the autotuner's pick), else 0.  No counterpart in the
 * reference. */
int rb_amg_level_fused_first(rb_amg ml, int level, int* fused);
/* The level from which the rest of the cycle runs as one cluster launch
 * (-1: none) and the CTAs of that cluster.  No counterpart in the
 * reference (it describes how this library schedules the cycle). */
int rb_amg_tail_info(rb_amg ml, int* start_level, int* ctas);
/* The cycle times (ms) the setup measured to pick that level: without the
 * cluster tail first, then for each qualifying start from the coarsest
 * upwards (empty when the choice came from the tune cache or was forced).
 * Writes min(*count, cap) values.  No counterpart in the reference. */
int rb_amg_tail_timings(rb_amg ml, double* ms, int cap, int* count);
/* Kernels this library has launched so far (graph replays count their
 * kernel nodes). */
int rb_launch_count(int64_t* count);
/* Device allocations (cudaMalloc) this library has made so far.  No
 * counterpart in the reference; a diagnostic for callers that audit
 * allocation-free paths. */
int rb_device_alloc_count(int64_t* count);

/* ||b - A x||_2 into norm_out[0] without allocating device memory.  No
 * counterpart in the reference.  For callers that must not allocate while
 * they run: runtimes that hand the solver a fixed memory budget and forbid
 * allocation once a solve is under way (an allocation there can fail), and
 * real-time loops in which cudaMalloc's implicit device synchronisation
 * would break the deadline.  Every pointer is device memory owned by the caller (CSR arrays of A
 * with n_rows rows, x, b, and one double for the result); stream is a
 * cudaStream_t (NULL = default stream).  Its scratch is a file-scope device
 * array (128 KiB per device, held until exit), so n_rows is limited to
 * 16777216 (RB_ERR_INVALID beyond).  The first call on a device resolves the
 * array's address and must precede any stream capture.  Calls share
 * the array: calls that overlap on the GPU race. */
int rb_residual_norm_noalloc(int n_rows, const int* rowptr, const int* cols, const double* vals,
                             const double* x, const double* b, double* norm_out, void* stream);

/* ------------------------------------------------------------------ Krylov */
#define RB_PCG_REFERENCE 0 /* par_cg.cpp:121-263 exactly: stop on r.z < tol*sqrt(b.Mb) */
#define RB_PCG_TRUE_RESIDUAL 1 /* stop on ||b - A x|| / ||b|| < tol */

/* PCG (krylov/par_cg.cpp:121-263).  When A is the matrix ml was set up with,
 * A p reads the hierarchy's copies of it (changing A's values after setup
 * needs a new setup).  hist receives the reference's history
 * (sqrt(r.z) then r.z/b.Mb) in RB_PCG_REFERENCE mode, ||r||/||b|| otherwise;
 * n_hist receives the entry count. */
int rb_pcg(rb_csr A, rb_amg ml, rb_vec x, rb_vec b, double tol, int max_iter, int mode,
           double* hist, int cap, int* n_hist);
/* --------------------------------------------------- differentiation */
/* Finite-volume assembly of -div(k grad u) on an nx x ny grid of unit cells
 * (cell c = y nx + x), homogeneous Dirichlet walls: face transmissibility
 * 2 k_i k_j / (k_i + k_j) between cells, 2 k_i to a wall; rows sorted by
 * column.  k is a device array of nx ny conductivities.  No counterpart in
 * the reference. */
int rb_fv_assemble(int nx, int ny, const double* k, rb_csr* A);
/* Backward of rb_fv_assemble: gk (device, nx ny) = dL/dk from gA (device,
 * one entry per stored entry of A) = dL/dA. */
int rb_fv_backward(int nx, int ny, const double* k, rb_csr A, const double* gA, double* gk);
/* SDDMM on A's pattern: out_j = scale lambda_i x_col(j) for every stored
 * entry j of row i (device arrays).  With scale = -1, lambda the adjoint
 * and x the primal solution this is dL/dA for x = A^-1 b. */
int rb_sddmm(rb_csr A, const double* lambda, const double* x, double scale, double* out);
/* A^T lambda = g through the hierarchy ml built for A: PCG when A is
 * symmetric (the transposed V-cycle is then the V-cycle itself), else
 * BiCGStab with the transposed cycle (A_l^T on every level, the same P and
 * R and smoother diagonals, Jacobi or L1-Jacobi smoothing).  lambda starts
 * from zero; iters and relres (may be NULL) receive the iterations and the
 * final true relative residual ||g - A^T lambda|| / ||g||. */
int rb_adjoint_solve(rb_csr A, rb_amg ml, rb_vec lambda, rb_vec g, double tol, int max_iter,
                     int* iters, double* relres);

/* ------------------------------------------------- batches of systems */
/* An uneven batch of independent systems (no counterpart in the reference).
 * Each matrix gets the hierarchy rb_amg_setup would build for it alone; the
 * levels are packed block-diagonally so one V-cycle of the batch is one
 * launch per operation for all systems, and rb_batch_pcg runs the
 * iterations of all systems on the device: one CUDA graph launch holds a
 * while loop over whole iterations, with per-system CG scalars, active
 * flags and stopping tests (true-residual confirmation included) kept on the
 * device.  Vectors of a batch are the systems' vectors concatenated in order
 * (rb_batch_offsets gives the first row of each). */
int rb_batch_setup(int n_sys, const rb_csr* mats, const rb_amg_opts* opts, rb_batch* out);
int rb_batch_destroy(rb_batch B);
/* number of systems, total rows, levels of the packed hierarchy */
int rb_batch_info(rb_batch B, int* n_sys, int64_t* total_rows, int* levels);
/* offsets[n_sys + 1] (first row of each system, then the total) and the
 * levels of each system's own hierarchy (levels[n_sys]); either may be NULL */
int rb_batch_offsets(rb_batch B, int64_t* offsets, int* levels);
/* x = M b: one V-cycle of every system from a zero guess */
int rb_batch_cycle(rb_batch B, rb_vec x, rb_vec b);
/* Preconditioned CG per system in true-residual mode; iters[n_sys] and
 * relres[n_sys] receive each system's iterations and final true relative
 * residual.  RB_ERR_NOT_CONVERGED if any system did not reach tol. */
int rb_batch_pcg(rb_batch B, rb_vec x, rb_vec b, double tol, int max_iter, int* iters,
                 double* relres);
/* Times the host waited on the device during the last rb_batch_pcg (one per
 * graph launch of its device-side loop; a launch ends at convergence,
 * breakdown, the iteration limit or a failed true-residual confirmation).
 * No counterpart in the reference. */
int rb_batch_host_waits(rb_batch B, int* waits);

/* One V-cycle from a zero guess applied to k columns at once, X = M B
 * (columns interleaved by row, n * k entries each; k in 2..32; Jacobi or
 * L1-Jacobi smoothing).  No counterpart in the reference. */
int rb_amg_cycle_block(rb_amg ml, rb_vec X, rb_vec B, int k);
/* k right-hand sides over one hierarchy (no counterpart in the reference,
 * which solves one at a time).  X and B are vectors of n * k entries with the
 * columns interleaved by row: entry (i, c) at i * k + c.  Runs k independent
 * preconditioned CG recurrences whose SpMMs read every matrix once for all
 * columns; each column stops when its true ||b_c - A x_c|| / ||b_c|| <= tol.
 * iters[k] and relres[k] (host) receive each column's iterations and final
 * true relative residual.  k in 1..32; the smoother must be Jacobi or
 * L1-Jacobi.  Columns with b_c = 0 are left as given. */
int rb_pcg_block(rb_csr A, rb_amg ml, rb_vec X, rb_vec B, int k, double tol, int max_iter,
                 int* iters, double* relres);
/* CG (krylov/par_cg.cpp:8-118); hist = ||r||/||b||. */
int rb_cg(rb_csr A, rb_vec x, rb_vec b, double tol, int max_iter, double* hist, int cap,
          int* n_hist);
/* BiCGStab (krylov/par_bicgstab.cpp:11-126) when ml is NULL, Pre_BiCGStab
 * (:240-371, right-preconditioned) otherwise; hist = ||r||. */
int rb_bicgstab(rb_csr A, rb_amg ml, rb_vec x, rb_vec b, double tol, int max_iter,
                double* hist, int cap, int* n_hist);

#ifdef __cplusplus
}
#endif
#endif
