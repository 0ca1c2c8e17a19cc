/*
 * raptor_oracle.c -- TEST INFRASTRUCTURE ONLY (see raptor_oracle.h).
 *
 * CPU restatement of RAPtor's AMG path at MPI world size 1.  Citations are
 * file:line within the reference project (13manan/raptor).  At world size 1
 * every ParCSRMatrix has an empty off_proc block, so only the on_proc loops
 * are restated.  Build with -ffp-contract=off: the reference's -O3 x86-64
 * build has no FMA, and bit-exact setup patterns depend on separate mul/add.
 */
#include "raptor_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ZERO_TOL 1e-16 /* core/types.hpp:26 */

/* row-parallel loops: a team only when more than one thread is asked for */
static int g_threads = 1;
void oc_set_threads(int n) { g_threads = n > 1 ? n : 1; }
int oc_get_threads(void) { return g_threads; }
#define OC_ROWS_PARALLEL _Pragma("omp parallel for num_threads(g_threads) if(g_threads > 1) schedule(static)")
#define OC_RAND_MAX 2147483647.0 /* glibc RAND_MAX used by par_strength.cpp:78 */

/* ------------------------------------------------------------------------ */
/* containers                                                               */
/* ------------------------------------------------------------------------ */

static oc_csr* csr_alloc(int n_rows, int n_cols, int cap) {
    oc_csr* A = (oc_csr*)calloc(1, sizeof(oc_csr));
    A->n_rows = n_rows;
    A->n_cols = n_cols;
    A->cap = cap > 0 ? cap : 1;
    A->rowptr = (int*)calloc((size_t)n_rows + 1, sizeof(int));
    A->cols = (int*)malloc((size_t)A->cap * sizeof(int));
    A->vals = (double*)malloc((size_t)A->cap * sizeof(double));
    return A;
}

static void csr_push(oc_csr* A, int col, double v) {
    if (A->nnz == A->cap) {
        A->cap *= 2;
        A->cols = (int*)realloc(A->cols, (size_t)A->cap * sizeof(int));
        A->vals = (double*)realloc(A->vals, (size_t)A->cap * sizeof(double));
    }
    A->cols[A->nnz] = col;
    A->vals[A->nnz] = v;
    A->nnz++;
}

oc_csr* oc_csr_new(int n_rows, int n_cols, int nnz, const int* rowptr,
                   const int* cols, const double* vals) {
    oc_csr* A = csr_alloc(n_rows, n_cols, nnz);
    memcpy(A->rowptr, rowptr, ((size_t)n_rows + 1) * sizeof(int));
    if (nnz) {
        memcpy(A->cols, cols, (size_t)nnz * sizeof(int));
        memcpy(A->vals, vals, (size_t)nnz * sizeof(double));
    }
    A->nnz = nnz;
    return A;
}

oc_csr* oc_csr_copy(const oc_csr* A) {
    return oc_csr_new(A->n_rows, A->n_cols, A->nnz, A->rowptr, A->cols, A->vals);
}

void oc_csr_free(oc_csr* A) {
    if (!A) return;
    free(A->rowptr);
    free(A->cols);
    free(A->vals);
    free(A);
}

void oc_csr_info(const oc_csr* A, int* n_rows, int* n_cols, int* nnz) {
    *n_rows = A->n_rows;
    *n_cols = A->n_cols;
    *nnz = A->nnz;
}

void oc_csr_export(const oc_csr* A, int* rowptr, int* cols, double* vals) {
    memcpy(rowptr, A->rowptr, ((size_t)A->n_rows + 1) * sizeof(int));
    if (A->nnz) {
        memcpy(cols, A->cols, (size_t)A->nnz * sizeof(int));
        memcpy(vals, A->vals, (size_t)A->nnz * sizeof(double));
    }
}

/* Sort each row by column (core/matrix.cpp sort_helper, :588-618).  Rows of
 * the matrices sorted here never hold duplicate columns except in
 * add/subtract, where at most two duplicates meet and IEEE addition is
 * commutative, so a stable insertion sort gives the reference's result. */
void oc_csr_sort(oc_csr* A) {
    for (int i = 0; i < A->n_rows; i++) {
        int s = A->rowptr[i], e = A->rowptr[i + 1];
        for (int j = s + 1; j < e; j++) {
            int c = A->cols[j];
            double v = A->vals[j];
            int k = j - 1;
            while (k >= s && A->cols[k] > c) {
                A->cols[k + 1] = A->cols[k];
                A->vals[k + 1] = A->vals[k];
                k--;
            }
            A->cols[k + 1] = c;
            A->vals[k + 1] = v;
        }
    }
}

/* Move the diagonal entry to the front of its row, shifting the entries
 * before it (core/matrix.cpp move_diag_helper, :730-786). */
void oc_csr_move_diag(oc_csr* A) {
    for (int i = 0; i < A->n_rows; i++) {
        int s = A->rowptr[i], e = A->rowptr[i + 1];
        for (int j = s; j < e; j++) {
            if (A->cols[j] == i) {
                double t = A->vals[j];
                for (int k = j; k > s; k--) {
                    A->cols[k] = A->cols[k - 1];
                    A->vals[k] = A->vals[k - 1];
                }
                A->cols[s] = i;
                A->vals[s] = t;
                break;
            }
        }
    }
}

/* Drop entries with |v| < 1e-16 after summing duplicates of a sorted row
 * (core/matrix.cpp remove_duplicates_helper for CSR, :923+). */
static void csr_remove_duplicates(oc_csr* A) {
    int out = 0;
    int orig_start = A->rowptr[0];
    for (int i = 0; i < A->n_rows; i++) {
        int orig_end = A->rowptr[i + 1];
        int row_start = out;
        int prev = -1;
        for (int j = orig_start; j < orig_end; j++) {
            int c = A->cols[j];
            if (out > row_start && c == prev) {
                A->vals[out - 1] += A->vals[j];
            } else {
                if (out > row_start && fabs(A->vals[out - 1]) < ZERO_TOL) out--;
                A->cols[out] = c;
                A->vals[out] = A->vals[j];
                out++;
                prev = c;
            }
        }
        if (out > row_start && fabs(A->vals[out - 1]) < ZERO_TOL) out--;
        orig_start = orig_end;
        A->rowptr[i + 1] = out;
    }
    A->nnz = out;
}

/* Stable transpose: column lists hold rows in increasing order
 * (core/matrix.cpp CSR_to_CSC, :492-538). */
oc_csr* oc_csr_transpose(const oc_csr* A) {
    oc_csr* T = csr_alloc(A->n_cols, A->n_rows, A->nnz);
    int* cnt = (int*)calloc((size_t)A->n_cols + 1, sizeof(int));
    for (int j = 0; j < A->nnz; j++) cnt[A->cols[j] + 1]++;
    for (int c = 0; c < A->n_cols; c++) cnt[c + 1] += cnt[c];
    memcpy(T->rowptr, cnt, ((size_t)A->n_cols + 1) * sizeof(int));
    for (int i = 0; i < A->n_rows; i++) {
        for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) {
            int c = A->cols[j];
            int p = cnt[c]++;
            T->cols[p] = i;
            T->vals[p] = A->vals[j];
        }
    }
    T->nnz = A->nnz;
    free(cnt);
    return T;
}

/* ------------------------------------------------------------------------ */
/* gallery                                                                  */
/* ------------------------------------------------------------------------ */

/* gallery/diffusion.hpp:58-85 */
void oc_diffusion_stencil_2d(double eps, double theta, double* st) {
    double C = cos(theta), S = sin(theta);
    double CS = C * S, CC = C * C, SS = S * S;
    double v1 = ((-1 * eps - 1) * CC + (-1 * eps - 1) * SS + (3 * eps - 3) * CS) / 6.0;
    double v2 = ((2 * eps - 4) * CC + (-4 * eps + 2) * SS) / 6.0;
    double v3 = ((-1 * eps - 1) * CC + (-1 * eps - 1) * SS + (-3 * eps + 3) * CS) / 6.0;
    double v4 = ((-4 * eps + 2) * CC + (2 * eps - 4) * SS) / 6.0;
    double v5 = ((8 * eps + 8) * CC + (8 * eps + 8) * SS) / 6.0;
    st[0] = v1; st[1] = v2; st[2] = v3; st[3] = v4; st[4] = v5;
    st[5] = v4; st[6] = v3; st[7] = v2; st[8] = v1;
}

/* gallery/laplacian27pt.hpp:27-37 */
void oc_laplace_stencil_27pt(double* st) {
    for (int i = 0; i < 27; i++) st[i] = -1;
    st[13] = 26;
}

/* gallery/par_stencil.hpp:16-236 at world size 1 (first_local_row = 0). */
oc_csr* oc_stencil_grid(const double* stencil, const int* grid, int dim) {
    int slen = 1;
    for (int d = 0; d < dim; d++) slen *= 3;
    long N = 1;
    for (int d = 0; d < dim; d++) N *= grid[d];
    int Ns = 0;
    for (int s = 0; s < slen; s++)
        if (fabs(stencil[s]) > ZERO_TOL) Ns++;
    int strides[8];
    strides[0] = 1;
    for (int i = 0; i < dim - 1; i++) strides[i + 1] = grid[dim - i - 1] * strides[i];
    int* idx = (int*)calloc((size_t)Ns * dim, sizeof(int)); /* idx[ctr*dim + j] */
    double* nzs = (double*)malloc(sizeof(double) * Ns);
    long* diags = (long*)calloc(Ns, sizeof(long));
    int ctr = 0;
    for (int s = 0; s < slen; s++) {
        if (fabs(stencil[s]) > ZERO_TOL) {
            int p = 1;
            for (int j = 0; j < dim; j++) {
                idx[ctr * dim + (dim - j - 1)] = ((s / p) % 3) - 1;
                p *= 3;
            }
            nzs[ctr] = stencil[s];
            ctr++;
        }
    }
    for (int i = 0; i < dim; i++)
        for (int j = 0; j < Ns; j++) diags[j] += (long)strides[i] * idx[j * dim + (dim - i - 1)];
    double* data = (double*)malloc(sizeof(double) * (size_t)Ns * N);
    for (int s = 0; s < Ns; s++)
        for (long r = 0; r < N; r++) data[(size_t)s * N + r] = nzs[s];
    long first = 0, last = N - 1;
    /* boundary masks, par_stencil.hpp:137-209 */
    for (int s = 0; s < Ns; s++) {
        size_t base = (size_t)s * N;
        for (int j = 0; j < dim; j++) {
            int o = idx[s * dim + j];
            if (o == 0) continue;
            long len = 1;
            for (int k = 0; k < dim - j - 1; k++) len *= grid[k];
            long step = len * grid[0];
            if (o > 0) {
                long cur = step * (first / step);
                for (long k = cur; k < last + 1; k += step) {
                    for (long l = 0; l < len; l++) {
                        if (k + l > last) break;
                        if (k + l < first) continue;
                        data[base + (k - first) + l] = 0;
                    }
                }
            } else {
                long cur = step * (((last - 1) / step) + 1);
                for (long k = cur; k > first; k -= step) {
                    for (long l = 0; l < len; l++) {
                        if (k - l - 1 < first) break;
                        else if (k - l - 1 > last) continue;
                        data[base + (k - l - first) - 1] = 0;
                    }
                }
            }
        }
    }
    /* rows, par_stencil.hpp:211-228 (value from the mirrored entry) */
    oc_csr* A = csr_alloc((int)N, (int)N, (int)(N * Ns));
    for (long i = 0; i < N; i++) {
        for (int d = 0; d < Ns; d++) {
            long col = diags[d] + i;
            double v = data[(size_t)(Ns - d - 1) * N + i];
            if (col >= 0 && col < N && fabs(v) > ZERO_TOL) csr_push(A, (int)col, v);
        }
        A->rowptr[i + 1] = A->nnz;
    }
    oc_csr_sort(A); /* finalize() sorts on_proc, par_matrix.cpp:111-114 */
    free(idx); free(nzs); free(diags); free(data);
    return A;
}

/* ------------------------------------------------------------------------ */
/* SpMV family (util/linalg/spmv.cpp)                                       */
/* ------------------------------------------------------------------------ */

/* CSR_spmv, spmv.cpp:52-67 */
void oc_spmv(const oc_csr* A, const double* x, double* b) {
    OC_ROWS_PARALLEL
    for (int i = 0; i < A->n_rows; i++) {
        double v = 0;
        for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) v += A->vals[j] * x[A->cols[j]];
        b[i] = v;
    }
}

/* CSR_residual, spmv.cpp:69-85 */
void oc_residual(const oc_csr* A, const double* x, const double* b, double* r) {
    OC_ROWS_PARALLEL
    for (int i = 0; i < A->n_rows; i++) {
        double v = b[i];
        for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) v -= A->vals[j] * x[A->cols[j]];
        r[i] = v;
    }
}

/* Matrix::mult_T zero fill + CSR_append_T, matrix.hpp:342-348, spmv.cpp:150-163 */
void oc_spmv_T(const oc_csr* A, const double* x, double* b) {
    for (int c = 0; c < A->n_cols; c++) b[c] = 0.0;
    for (int i = 0; i < A->n_rows; i++)
        for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) b[A->cols[j]] += A->vals[j] * x[i];
}

/* CSR_append, spmv.cpp:88-103 */
void oc_spmv_append(const oc_csr* A, const double* x, double* b) {
    OC_ROWS_PARALLEL
    for (int i = 0; i < A->n_rows; i++) {
        double v = 0;
        for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) v += A->vals[j] * x[A->cols[j]];
        b[i] += v;
    }
}

/* ------------------------------------------------------------------------ */
/* block CSR (BSRMatrix, core/matrix.hpp:962-1060)                          */
/* nbr x nbc blocks of br x bc values; block j's values at vals[j*br*bc],   */
/* row-major (the reference's block_vals[j][r*bc + c]).                     */
/* ------------------------------------------------------------------------ */

/* BSR_spmv, spmv.cpp:121-148 */
void oc_bsr_spmv(int nbr, int br, int bc, const int* rowptr, const int* cols,
                 const double* vals, const double* x, double* b) {
    const size_t bs = (size_t)br * bc;
    for (int i = 0; i < nbr; i++) {
        const int first_row = i * br;
        for (int row = 0; row < br; row++) {
            double val = 0;
            const size_t idx = (size_t)row * bc;
            for (int j = rowptr[i]; j < rowptr[i + 1]; j++) {
                const size_t first_col = (size_t)cols[j] * bc;
                const double* block = vals + (size_t)j * bs;
                for (int col = 0; col < bc; col++) val += block[idx + col] * x[first_col + col];
            }
            b[first_row + row] = val;
        }
    }
}

/* BSR_append with the block Matrix::append, spmv.cpp:105-119,
 * matrix.hpp:287-298; neg != 0: the block append_neg (matrix.hpp:313-324) */
static void bsr_append_sign(int nbr, int br, int bc, const int* rowptr, const int* cols,
                            const double* vals, const double* x, double* b, int neg) {
    const size_t bs = (size_t)br * bc;
    for (int i = 0; i < nbr; i++)
        for (int j = rowptr[i]; j < rowptr[i + 1]; j++) {
            const size_t first_row = (size_t)i * br, first_col = (size_t)cols[j] * bc;
            const double* block = vals + (size_t)j * bs;
            for (int row = 0; row < br; row++)
                for (int col = 0; col < bc; col++) {
                    if (neg)
                        b[first_row + row] -= block[row * bc + col] * x[first_col + col];
                    else
                        b[first_row + row] += block[row * bc + col] * x[first_col + col];
                }
        }
}

void oc_bsr_append(int nbr, int br, int bc, const int* rowptr, const int* cols,
                   const double* vals, const double* x, double* b) {
    bsr_append_sign(nbr, br, bc, rowptr, cols, vals, x, b, 0);
}

/* BSRMatrix::spmv_residual, spmv.cpp:363-368 */
void oc_bsr_residual(int nbr, int br, int bc, const int* rowptr, const int* cols,
                     const double* vals, const double* x, const double* b, double* r) {
    for (size_t i = 0; i < (size_t)nbr * br; i++) r[i] = b[i];
    bsr_append_sign(nbr, br, bc, rowptr, cols, vals, x, r, 1);
}

/* Matrix::mult_T zero fill (matrix.hpp:342-348), then CSR_append_T over the
 * blocks (spmv.cpp:150-163) with the block append_T (matrix.hpp:299-312) */
void oc_bsr_spmv_T(int nbr, int nbc, int br, int bc, const int* rowptr, const int* cols,
                   const double* vals, const double* x, double* b) {
    const size_t bs = (size_t)br * bc;
    for (size_t c = 0; c < (size_t)nbc * bc; c++) b[c] = 0.0;
    for (int i = 0; i < nbr; i++)
        for (int j = rowptr[i]; j < rowptr[i + 1]; j++) {
            const size_t first_row = (size_t)i * br, first_col = (size_t)cols[j] * bc;
            const double* block = vals + (size_t)j * bs;
            for (int row = 0; row < br; row++) {
                const double x_val = x[first_row + row];
                for (int col = 0; col < bc; col++)
                    b[first_col + col] += block[row * bc + col] * x_val;
            }
        }
}

/* BSR_to_CSR, core/matrix.cpp:358-395: scalar rows in order, a row's blocks
 * in storage order, a block row's columns in order, |v| > zero_tol kept */
oc_csr* oc_bsr_to_csr(int nbr, int nbc, int br, int bc, const int* rowptr, const int* cols,
                      const double* vals) {
    const size_t bs = (size_t)br * bc;
    oc_csr* B = csr_alloc(nbr * br, nbc * bc, rowptr[nbr] > 0 ? rowptr[nbr] : 1);
    for (int i = 0; i < nbr; i++)
        for (int row = 0; row < br; row++) {
            for (int j = rowptr[i]; j < rowptr[i + 1]; j++)
                for (int col = 0; col < bc; col++) {
                    const double v = vals[(size_t)j * bs + (size_t)row * bc + col];
                    if (fabs(v) > ZERO_TOL) csr_push(B, cols[j] * bc + col, v);
                }
            B->rowptr[i * br + row + 1] = B->nnz;
        }
    return B;
}

/* ------------------------------------------------------------------------ */
/* strength of connection (par_strength.cpp)                                */
/* ------------------------------------------------------------------------ */

/* classical_strength, par_strength.cpp:8-339 (num_variables = 1).
 * A must be sorted with the diagonal first. */
oc_csr* oc_classical_strength(const oc_csr* A, double theta) {
    oc_csr* S = csr_alloc(A->n_rows, A->n_cols, A->nnz);
    for (int i = 0; i < A->n_rows; i++) {
        int rs = A->rowptr[i], re = A->rowptr[i + 1];
        if (re - rs) {
            double diag, row_scale;
            if (A->cols[rs] == i) { diag = A->vals[rs]; rs++; }
            else diag = 0.0;
            if (diag < 0.0) {
                row_scale = -OC_RAND_MAX;
                for (int j = rs; j < re; j++) if (A->vals[j] > row_scale) row_scale = A->vals[j];
            } else {
                row_scale = OC_RAND_MAX;
                for (int j = rs; j < re; j++) if (A->vals[j] < row_scale) row_scale = A->vals[j];
            }
            double threshold = row_scale * theta;
            csr_push(S, i, diag);
            for (int j = rs; j < re; j++) {
                double v = A->vals[j];
                if (diag < 0 ? (v > threshold) : (v < threshold)) csr_push(S, A->cols[j], v);
            }
        }
        S->rowptr[i + 1] = S->nnz;
    }
    return S;
}

/* symmetric_strength, par_strength.cpp:342-531 */
oc_csr* oc_symmetric_strength(const oc_csr* A, double theta) {
    int n = A->n_rows;
    double* row_scales = (double*)calloc(n, sizeof(double));
    int* neg = (int*)calloc(n, sizeof(int));
    for (int i = 0; i < n; i++) {
        int rs = A->rowptr[i], re = A->rowptr[i + 1];
        if (re - rs) {
            double diag, row_scale;
            if (A->cols[rs] == i) { diag = A->vals[rs]; rs++; }
            else diag = 0.0;
            if (diag < 0.0) {
                neg[i] = 1;
                row_scale = -OC_RAND_MAX;
                for (int j = rs; j < re; j++) if (A->vals[j] > row_scale) row_scale = A->vals[j];
            } else {
                neg[i] = 0;
                row_scale = OC_RAND_MAX;
                for (int j = rs; j < re; j++) if (A->vals[j] < row_scale) row_scale = A->vals[j];
            }
            row_scales[i] = row_scale * theta;
        }
    }
    oc_csr* S = csr_alloc(n, A->n_cols, A->nnz);
    for (int i = 0; i < n; i++) {
        int rs = A->rowptr[i], re = A->rowptr[i + 1];
        if (re - rs) {
            int nd = neg[i];
            double thr = row_scales[i];
            csr_push(S, i, A->vals[rs++]); /* the first entry is taken as the diagonal */
            for (int j = rs; j < re; j++) {
                double v = A->vals[j];
                int c = A->cols[j];
                if ((nd && v > thr) || (!nd && v < thr) || (neg[c] && v > row_scales[c]) ||
                    (!neg[c] && v < row_scales[c]))
                    csr_push(S, c, v);
            }
        }
        S->rowptr[i + 1] = S->nnz;
    }
    free(row_scales);
    free(neg);
    return S;
}

/* ------------------------------------------------------------------------ */
/* PMIS C/F splitting (ruge_stuben/par_cf_splitting.cpp)                    */
/* ------------------------------------------------------------------------ */

/* Column lists of S without each row's leading diagonal
 * (transpose, par_cf_splitting.cpp:158-244). */
static void s_transpose(const oc_csr* S, int** colptr_out, int** colidx_out) {
    int n = S->n_rows, nc = S->n_cols;
    int* cp = (int*)calloc((size_t)nc + 1, sizeof(int));
    int* ci = (int*)malloc(sizeof(int) * (S->nnz + 1));
    for (int i = 0; i < n; i++) {
        int s = S->rowptr[i], e = S->rowptr[i + 1];
        if (s < e && S->cols[s] == i) s++;
        for (int j = s; j < e; j++) cp[S->cols[j] + 1]++;
    }
    for (int c = 0; c < nc; c++) cp[c + 1] += cp[c];
    int* fill = (int*)calloc(nc, sizeof(int));
    for (int i = 0; i < n; i++) {
        int s = S->rowptr[i], e = S->rowptr[i + 1];
        if (s < e && S->cols[s] == i) s++;
        for (int j = s; j < e; j++) {
            int c = S->cols[j];
            ci[cp[c] + fill[c]++] = i;
        }
    }
    free(fill);
    *colptr_out = cp;
    *colidx_out = ci;
}

/* split_pmis (:75-89) -> set_initial_states (:114-131) -> pmis_main_loop
 * (:1229-1381) with initial_weights (:246-309), select_independent_set
 * (:403-495) and update_states (:1200-1227).  Off-process parts are empty. */
void oc_split_pmis(const oc_csr* S, const double* rand_vals, int* states) {
    int n = S->n_rows;
    for (int i = 0; i < n; i++) {
        int len = S->rowptr[i + 1] - S->rowptr[i];
        states[i] = len > 1 ? OC_UNASSIGNED : OC_NONEIGHBORS;
    }
    int *cp, *ci;
    s_transpose(S, &cp, &ci);
    double* w = (double*)malloc(sizeof(double) * (n + 1));
    for (int i = 0; i < n; i++) w[i] = rand_vals[i];
    for (int i = 0; i < n; i++) {
        int s = S->rowptr[i], e = S->rowptr[i + 1];
        if (s < e && S->cols[s] == i) s++;
        for (int j = s; j < e; j++) w[S->cols[j]] += 1;
    }
    int* un = (int*)malloc(sizeof(int) * (n + 1));
    int* newc = (int*)malloc(sizeof(int) * (n + 1));
    int rem = 0;
    for (int i = 0; i < n; i++) {
        if (states[i] == OC_UNASSIGNED && w[i] < 1) { states[i] = OC_UNSELECTED; w[i] = 0.0; }
        else if (states[i] == OC_UNASSIGNED) un[rem++] = i;
        else w[i] = 0.0;
    }
    int first_pass = 1;
    while (rem || first_pass) {
        int nnew = 0;
        for (int t = 0; t < rem; t++) {
            int u = un[t];
            double wu = w[u];
            int s = S->rowptr[u], e = S->rowptr[u + 1], j;
            if (s < e && S->cols[s] == u) s++;
            for (j = s; j < e; j++) if (w[S->cols[j]] > wu) break;
            if (j != e) continue;
            for (j = cp[u]; j < cp[u + 1]; j++) if (w[ci[j]] > wu) break;
            if (j != cp[u + 1]) continue;
            states[u] = OC_NEWSELECTION;
            newc[nnew++] = u;
        }
        for (int t = 0; t < nnew; t++) {
            int c = newc[t];
            for (int j = cp[c]; j < cp[c + 1]; j++)
                if (states[ci[j]] == OC_UNASSIGNED) states[ci[j]] = OC_NEWUNSELECTION;
        }
        int k = 0;
        for (int t = 0; t < rem; t++) {
            int u = un[t];
            if (states[u] == OC_NEWSELECTION) { w[u] = 0.0; states[u] = OC_SELECTED; }
            else if (w[u] < 1.0 || states[u] == OC_NEWUNSELECTION) { w[u] = 0.0; states[u] = OC_UNSELECTED; }
            else un[k++] = u;
        }
        rem = k;
        first_pass = 0;
    }
    free(cp); free(ci); free(w); free(un); free(newc);
}

/* ------------------------------------------------------------------------ */
/* interpolation (ruge_stuben/par_interpolation.cpp)                        */
/* ------------------------------------------------------------------------ */

/* split_rs, ruge_stuben/cf_splitting.cpp:277-322: weights are the column
 * counts of S (diagonal left out), rs_first_pass (:69-209) visits the points
 * from the largest weight down through weight buckets (weight_ptr /
 * weight_sizes / weight_idx_to_col / col_to_weight_idx, restated with the
 * same moves so that ties resolve identically): an unassigned point becomes
 * C, the unassigned points it influences become F and each unassigned
 * strong neighbour of those gains weight, and the unassigned points that
 * influence it lose weight; rs_second_pass (:211-275) promotes an F point to
 * C when a strong F neighbour shares no C point with it.  prev_states keeps
 * the caller's states (the parallel driver sets NoNeighbors first,
 * par_cf_splitting.cpp:7-30 -> set_initial_states :114-131); otherwise every
 * point starts unassigned.  HMIS and Falgout at world size 1 reduce to this:
 * the first pass only, resp. both passes, followed by PMIS / CLJP loops that
 * find nothing left to assign (par_cf_splitting.cpp:50-112). */
void oc_split_rs(const oc_csr* S, int* states, int prev_states, int second_pass) {
    int n = S->n_rows, nc = S->n_cols;
    int *colptr, *colidx;
    s_transpose(S, &colptr, &colidx);
    if (!prev_states)
        for (int i = 0; i < n; i++) states[i] = OC_UNASSIGNED;
    int* w = (int*)malloc(sizeof(int) * ((size_t)nc + 1));
    int* wptr = (int*)calloc((size_t)nc + 2, sizeof(int));
    int* wsz = (int*)calloc((size_t)nc + 1, sizeof(int));
    int* w2c = (int*)malloc(sizeof(int) * ((size_t)nc + 1));
    int* c2w = (int*)malloc(sizeof(int) * ((size_t)nc + 1));
    for (int i = 0; i < nc; i++) w[i] = colptr[i + 1] - colptr[i];
    for (int i = 0; i < nc; i++) wsz[w[i]]++;
    wptr[0] = 0;
    for (int i = 0; i < nc; i++) {
        wptr[i + 1] = wptr[i] + wsz[i];
        wsz[i] = 0;
    }
    for (int i = 0; i < nc; i++) {
        int wt = w[i];
        int idx = wptr[wt] + wsz[wt]++;
        w2c[idx] = i;
        c2w[i] = idx;
    }
    for (int i = nc - 1; i >= 0; i--) {
        int col = w2c[i];
        wsz[w[col]]--;
        if (states[col] != OC_UNASSIGNED) continue;
        states[col] = OC_SELECTED;
        for (int j = colptr[col]; j < colptr[col + 1]; j++) {
            int idx = colidx[j];
            if (states[idx] != OC_UNASSIGNED) continue;
            states[idx] = OC_UNSELECTED;
            int s = S->rowptr[idx], e = S->rowptr[idx + 1];
            if (s < e && S->cols[s] == idx) s++;
            for (int k = s; k < e; k++) {
                int idx_k = S->cols[k];
                if (states[idx_k] != OC_UNASSIGNED) continue;
                int wk = w[idx_k];
                if (wk >= nc - 1) continue;
                int old_pos = c2w[idx_k];
                int new_pos = wptr[wk] + wsz[wk] - 1;
                c2w[w2c[old_pos]] = new_pos;
                c2w[w2c[new_pos]] = old_pos;
                int t = w2c[old_pos]; w2c[old_pos] = w2c[new_pos]; w2c[new_pos] = t;
                wsz[wk] -= 1;
                wsz[wk + 1] += 1;
                wptr[wk + 1] = new_pos;
                w[idx_k]++;
            }
        }
        int s = S->rowptr[col], e = S->rowptr[col + 1];
        if (s < e && S->cols[s] == col) s++;
        for (int j = s; j < e; j++) {
            int idx = S->cols[j];
            if (states[idx] != OC_UNASSIGNED) continue;
            int wt = w[idx];
            if (wt == 0) continue;
            int old_pos = c2w[idx];
            int new_pos = wptr[wt];
            c2w[w2c[old_pos]] = new_pos;
            c2w[w2c[new_pos]] = old_pos;
            int t = w2c[old_pos]; w2c[old_pos] = w2c[new_pos]; w2c[new_pos] = t;
            wsz[wt] -= 1;
            wsz[wt - 1] += 1;
            wptr[wt] += 1;
            wptr[wt - 1] = wptr[wt] - wsz[wt - 1];
            w[idx]--;
        }
    }
    if (second_pass) {
        int* row_coarse = (int*)malloc(sizeof(int) * ((size_t)n + 1));
        for (int i = 0; i < n; i++) row_coarse[i] = -1;
        for (int i = 0; i < n; i++) {
            if (states[i] == OC_SELECTED) continue;
            int s = S->rowptr[i], e = S->rowptr[i + 1];
            for (int j = s; j < e; j++)
                if (states[S->cols[j]] == OC_SELECTED) row_coarse[S->cols[j]] = i;
            for (int j = s; j < e; j++) {
                int col = S->cols[j];
                if (states[col] != OC_UNSELECTED) continue;
                int sk = S->rowptr[col], ek = S->rowptr[col + 1];
                if (sk == ek) continue;
                int connection = 0;
                for (int k = sk; k < ek; k++)
                    if (row_coarse[S->cols[k]] == i) { connection = 1; break; }
                if (!connection) {
                    row_coarse[col] = i;
                    states[col] = OC_SELECTED;
                }
            }
        }
        free(row_coarse);
    }
    free(colptr); free(colidx); free(w); free(wptr); free(wsz); free(w2c); free(c2w);
}

/* split_cljp, ruge_stuben/cf_splitting.cpp:649-675 -> cljp_main_loop
 * (:479-545): weights = rand_vals + the number of rows in which a point is a
 * strong column; each round selects every unassigned point whose weight is
 * not exceeded by a strong neighbour in its row or its column
 * (select_independent_set, :324-378), removes the edges those new C points
 * satisfy (update_weights, :380-447; edgemark per nonzero of S, c_dep_cache
 * per point) and retires new C points and points whose weight fell below 1
 * (update_states, :449-477).  S is sorted with the diagonal first; its
 * column pattern leaves the diagonal out (transpose, :9-67). */
void oc_split_cljp(const oc_csr* S, const double* rand_vals, int* states) {
    int n = S->n_rows;
    int *colptr, *colidx;
    s_transpose(S, &colptr, &colidx);
    double* w = (double*)malloc(sizeof(double) * ((size_t)n + 1));
    int* unassigned = (int*)malloc(sizeof(int) * ((size_t)n + 1));
    int* newc = (int*)malloc(sizeof(int) * ((size_t)n + 1));
    int* cdep = (int*)calloc((size_t)n + 1, sizeof(int));
    char* edgemark = (char*)malloc((size_t)S->nnz + 1);
    memset(edgemark, 1, (size_t)S->nnz + 1);
    for (int i = 0; i < n; i++) {
        w[i] = rand_vals[i];
        unassigned[i] = i;
        states[i] = OC_UNASSIGNED;
    }
    for (int i = 0; i < n; i++) {
        int s = S->rowptr[i], e = S->rowptr[i + 1];
        if (s < e && S->cols[s] == i) s++;
        for (int j = s; j < e; j++) w[S->cols[j]] += 1;
    }
    int remaining = n;
    while (remaining) {
        int nnew = 0;
        for (int k = 0; k < remaining; k++) {
            int u = unassigned[k], j;
            double weight = w[u];
            int s = S->rowptr[u], e = S->rowptr[u + 1];
            if (s < e && S->cols[s] == u) s++;
            for (j = s; j < e; j++)
                if (w[S->cols[j]] > weight) break;
            if (j != e) continue;
            for (j = colptr[u]; j < colptr[u + 1]; j++)
                if (w[colidx[j]] > weight) break;
            if (j != colptr[u + 1]) continue;
            states[u] = OC_NEWSELECTION;
            newc[nnew++] = u;
        }
        for (int k = 0; k < nnew; k++) {
            int c = newc[k];
            int s = S->rowptr[c], e = S->rowptr[c + 1];
            if (s < e && S->cols[s] == c) s++;
            for (int j = s; j < e; j++) {
                int idx = S->cols[j];
                if (states[idx] == OC_UNASSIGNED && edgemark[j]) {
                    edgemark[j] = 0;
                    w[idx]--;
                }
            }
        }
        for (int k = 0; k < nnew; k++) {
            int c = newc[k];
            for (int j = colptr[c]; j < colptr[c + 1]; j++) {
                int idx = colidx[j];
                if (states[idx] == OC_UNASSIGNED) cdep[idx] = c;
            }
            for (int j = colptr[c]; j < colptr[c + 1]; j++) {
                int idx = colidx[j];
                if (states[idx] == OC_SELECTED) continue;
                int s = S->rowptr[idx], e = S->rowptr[idx + 1];
                if (s < e && S->cols[s] == idx) s++;
                for (int q = s; q < e; q++) {
                    int idx_k = S->cols[q];
                    if (states[idx_k] == OC_UNASSIGNED && edgemark[q] && cdep[idx_k] == c) {
                        edgemark[q] = 0;
                        w[idx_k]--;
                    }
                }
            }
        }
        int ctr = 0;
        for (int k = 0; k < remaining; k++) {
            int u = unassigned[k];
            if (states[u] == OC_NEWSELECTION) {
                w[u] = 0.0;
                states[u] = OC_SELECTED;
            } else if (w[u] < 1.0) {
                w[u] = 0.0;
                states[u] = OC_UNSELECTED;
            } else {
                unassigned[ctr++] = u;
            }
        }
        remaining = ctr;
    }
    free(colptr); free(colidx); free(w); free(unassigned); free(newc); free(cdep); free(edgemark);
}

static int* coarse_index(const int* states, int n, int* nc_out) {
    int* map = (int*)malloc(sizeof(int) * (n + 1));
    int nc = 0;
    for (int i = 0; i < n; i++) map[i] = states[i] == OC_SELECTED ? nc++ : -1;
    *nc_out = nc;
    return map;
}

/* direct_interpolation, par_interpolation.cpp:1453-1715 (world size 1).
 * A and S are sorted with the diagonal first (:1466-1469).  For an F row the
 * A values at the row's strong positions are found by walking A's row in
 * step with S's (:1476-1490); the strong C neighbours' values are summed by
 * sign, all off-diagonal values of A likewise, and each strong C neighbour
 * gets -(sum_all / sum_strong) / a_ii of its sign times its value.  With no
 * positive strong C neighbour the positive off-diagonal sum is lumped into
 * the diagonal (:1656-1660).  A row without a negative strong C neighbour
 * divides by zero there, as the reference does (:1645), but emits no entry
 * that uses the quotient. */
oc_csr* oc_direct_interp(const oc_csr* A, const oc_csr* S, const int* states) {
    int n = A->n_rows, nc;
    int* c2n = coarse_index(states, n, &nc);
    oc_csr* P = csr_alloc(n, nc, S->nnz + n);
    double* sa = (double*)malloc(sizeof(double) * ((size_t)S->nnz + 1));
    for (int i = 0; i < n; i++) {
        int ctr = A->rowptr[i], a1 = A->rowptr[i + 1];
        for (int j = S->rowptr[i]; j < S->rowptr[i + 1]; j++) {
            while (ctr < a1 && A->cols[ctr] != S->cols[j]) ctr++;
            sa[j] = ctr < a1 ? A->vals[ctr] : 0.0;
        }
    }
    for (int i = 0; i < n; i++) {
        if (states[i] == OC_SELECTED) {
            csr_push(P, c2n[i], 1);
            P->rowptr[i + 1] = P->nnz;
            continue;
        }
        double sum_strong_pos = 0, sum_strong_neg = 0, sum_all_pos = 0, sum_all_neg = 0;
        int start = S->rowptr[i], end = S->rowptr[i + 1], nstrong = 0;
        if (start < end && S->cols[start] == i) start++;
        for (int j = start; j < end; j++) {
            if (states[S->cols[j]] == OC_SELECTED) {
                double val = sa[j];
                if (val < 0) sum_strong_neg += val;
                else sum_strong_pos += val;
                nstrong++;
            }
        }
        if (nstrong == 0) {   /* no entry (and A's row may be empty) */
            P->rowptr[i + 1] = P->nnz;
            continue;
        }
        int a0 = A->rowptr[i], a1 = A->rowptr[i + 1];
        double diag = a0 < a1 ? A->vals[a0] : 0.0;
        for (int j = a0 + 1; j < a1; j++) {
            double val = A->vals[j];
            if (val < 0) sum_all_neg += val;
            else sum_all_pos += val;
        }
        double alpha = sum_all_neg / sum_strong_neg, beta;
        if (sum_strong_pos == 0) {
            diag += sum_all_pos;
            beta = 0;
        } else {
            beta = sum_all_pos / sum_strong_pos;
        }
        double neg_coeff = -alpha / diag;
        double pos_coeff = -beta / diag;
        for (int j = start; j < end; j++) {
            int col = S->cols[j];
            if (states[col] == OC_SELECTED) {
                double val = sa[j];
                csr_push(P, c2n[col], val < 0 ? neg_coeff * val : pos_coeff * val);
            }
        }
        P->rowptr[i + 1] = P->nnz;
    }
    free(sa);
    free(c2n);
    return P;
}

/* mod_classical_interpolation, par_interpolation.cpp:991-1451.
 * A and S are sorted with the diagonal first.  pos[] marks the positions of
 * row i's strong C neighbours; entries of earlier rows are < row start. */
oc_csr* oc_mod_classical_interp(const oc_csr* A, const oc_csr* S, const int* states) {
    int n = A->n_rows, nc;
    int* c2n = coarse_index(states, n, &nc);
    oc_csr* P = csr_alloc(n, nc, S->nnz + n);
    int* pos = (int*)malloc(sizeof(int) * (n + 1));
    for (int i = 0; i < n; i++) pos[i] = -1;
    for (int i = 0; i < n; i++) {
        if (states[i] == OC_SELECTED) {
            csr_push(P, c2n[i], 1);
            P->rowptr[i + 1] = P->nnz;
            continue;
        }
        int row_start = P->rowptr[i];
        for (int j = S->rowptr[i] + 1; j < S->rowptr[i + 1]; j++) {
            int c = S->cols[j];
            if (states[c] == OC_SELECTED) {
                pos[c] = P->nnz;
                csr_push(P, c2n[c], S->vals[j]);
            }
        }
        int start = A->rowptr[i], end = A->rowptr[i + 1];
        int ctr = S->rowptr[i] + 1, end_S = S->rowptr[i + 1];
        double weak_sum = A->vals[start++];
        for (int j = start; j < end; j++) {
            int col = A->cols[j];
            double val = A->vals[j];
            if (ctr < end_S && S->cols[ctr] == col) {
                ctr++;
                if (states[col] == OC_SELECTED) continue;
                double coarse_sum = 0;
                int sk = A->rowptr[col], ek = A->rowptr[col + 1];
                double diag = A->vals[sk++];
                int sign = diag > 0 ? 1 : -1;
                for (int k = sk; k < ek; k++) {
                    int ck = A->cols[k];
                    if (states[ck] == OC_SELECTED) {
                        double vk = A->vals[k];
                        if (vk * sign < 0 && pos[ck] >= row_start) coarse_sum += vk;
                    }
                }
                if (fabs(coarse_sum) < ZERO_TOL) weak_sum += val;
                else coarse_sum = val / coarse_sum;
                if (coarse_sum != 0.0) {
                    for (int k = A->rowptr[col] + 1; k < ek; k++) {
                        int ck = A->cols[k];
                        if (states[ck] == OC_SELECTED) {
                            double vk = A->vals[k];
                            int idx = pos[ck];
                            if (vk * sign < 0 && idx >= row_start) P->vals[idx] += coarse_sum * vk;
                        }
                    }
                }
            } else if (states[col] != OC_NONEIGHBORS) {
                weak_sum += val;
            }
        }
        P->rowptr[i + 1] = P->nnz;
        for (int j = P->rowptr[i]; j < P->rowptr[i + 1]; j++) P->vals[j] /= -weak_sum;
    }
    free(pos);
    free(c2n);
    return P;
}

/* filter_interp, par_interpolation.cpp:175-278 */
static void filter_interp(oc_csr* P, double thr) {
    if (!(thr > ZERO_TOL && thr <= 1)) return;
    int out = 0, rs = 0;
    for (int i = 0; i < P->n_rows; i++) {
        int re = P->rowptr[i + 1];
        int prev = out;
        double row_max = 0;
        for (int j = rs; j < re; j++) {
            double a = fabs(P->vals[j]);
            if (a > row_max) row_max = a;
        }
        row_max *= thr;
        double row_sum = 0, remain_sum = 0;
        for (int j = rs; j < re; j++) {
            double v = P->vals[j];
            row_sum += v;
            if (fabs(v) >= row_max) {
                P->cols[out] = P->cols[j];
                P->vals[out] = v;
                out++;
                remain_sum += v;
            }
        }
        if (fabs(remain_sum) > ZERO_TOL && fabs(row_sum - remain_sum) > ZERO_TOL) {
            double scale = row_sum / remain_sum;
            for (int j = prev; j < out; j++) P->vals[j] *= scale;
        }
        P->rowptr[i + 1] = out;
        rs = re;
    }
    P->nnz = out;
}

/* extended_interpolation (extended+i), par_interpolation.cpp:280-989, then
 * filter_interp (:946). */
oc_csr* oc_extended_interp(const oc_csr* A, const oc_csr* S, const int* states,
                           double filter) {
    int n = A->n_rows, nc;
    int* c2n = coarse_index(states, n, &nc);
    oc_csr* P = csr_alloc(n, nc, 4 * S->nnz + n);
    int* pos = (int*)malloc(sizeof(int) * (n + 1));
    for (int i = 0; i < n; i++) pos[i] = -1;
    for (int i = 0; i < n; i++) {
        if (states[i] != OC_UNSELECTED) {
            if (states[i] == OC_SELECTED) csr_push(P, c2n[i], 1);
            P->rowptr[i + 1] = P->nnz;
            continue;
        }
        int row_start = P->nnz;
        for (int j = S->rowptr[i] + 1; j < S->rowptr[i + 1]; j++) {
            int c = S->cols[j];
            if (states[c] == OC_SELECTED) {
                if (pos[c] < row_start) { pos[c] = P->nnz; csr_push(P, c2n[c], 0.0); }
            } else if (states[c] == OC_UNSELECTED) {
                for (int k = S->rowptr[c] + 1; k < S->rowptr[c + 1]; k++) {
                    int ck = S->cols[k];
                    if (states[ck] == OC_SELECTED && pos[ck] < row_start) {
                        pos[ck] = P->nnz;
                        csr_push(P, c2n[ck], 0.0);
                    }
                }
            }
        }
        pos[i] = P->nnz;
        int row_end = P->nnz;
        int start = A->rowptr[i], end = A->rowptr[i + 1];
        double weak_sum = A->vals[start++];
        int ctr = S->rowptr[i] + 1, end_S = S->rowptr[i + 1];
        for (int j = start; j < end; j++) {
            int col = A->cols[j];
            double val = A->vals[j];
            int idx = pos[col];
            if (idx >= row_start) {
                P->vals[idx] += val;
                if (ctr < end_S && S->cols[ctr] == col) ctr++;
            } else if (ctr < end_S && S->cols[ctr] == col) {
                ctr++;
                if (states[col] != OC_UNSELECTED) continue;
                double col_sum = 0;
                int sk = A->rowptr[col], ek = A->rowptr[col + 1];
                double diag = A->vals[sk++];
                int sign = diag > 0 ? 1 : -1;
                for (int k = sk; k < ek; k++) {
                    double vk = A->vals[k];
                    if (vk * sign < 0 && pos[A->cols[k]] >= row_start) col_sum += vk;
                }
                if (fabs(col_sum) < ZERO_TOL) {
                    weak_sum += val;
                } else {
                    col_sum = val / col_sum;
                    for (int k = A->rowptr[col] + 1; k < ek; k++) {
                        int ck = A->cols[k];
                        double vk = A->vals[k];
                        int id = pos[ck];
                        if (vk * sign < 0 && id >= row_start) {
                            if (ck == i) weak_sum += col_sum * vk;
                            else P->vals[id] += col_sum * vk;
                        }
                    }
                }
            } else {
                if (states[col] != OC_NONEIGHBORS) weak_sum += val;
            }
        }
        if (fabs(weak_sum) > ZERO_TOL)
            for (int j = row_start; j < row_end; j++) P->vals[j] /= -weak_sum;
        pos[i] = -1;
        P->rowptr[i + 1] = row_end;
    }
    filter_interp(P, filter);
    free(pos);
    free(c2n);
    return P;
}

/* ------------------------------------------------------------------------ */
/* SpGEMM and the Galerkin product                                          */
/* ------------------------------------------------------------------------ */

/* spgemm_helper, util/linalg/matmult.cpp:71-137: Gustavson with a linked
 * list; a row is emitted newest-first and |sum| <= 1e-16 is dropped. */
oc_csr* oc_spgemm(const oc_csr* A, const oc_csr* B) {
    int nb = B->n_cols;
    int* next = (int*)malloc(sizeof(int) * (nb + 1));
    double* sums = (double*)calloc((size_t)nb + 1, sizeof(double));
    for (int c = 0; c < nb; c++) next[c] = -1;
    oc_csr* C = csr_alloc(A->n_rows, nb, A->nnz + 16);
    for (int i = 0; i < A->n_rows; i++) {
        int head = -2, length = 0;
        for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) {
            int ca = A->cols[j];
            double va = A->vals[j];
            for (int k = B->rowptr[ca]; k < B->rowptr[ca + 1]; k++) {
                int cb = B->cols[k];
                sums[cb] += va * B->vals[k];
                if (next[cb] == -1) { next[cb] = head; head = cb; length++; }
            }
        }
        for (int t = 0; t < length; t++) {
            if (fabs(sums[head]) > ZERO_TOL) csr_push(C, head, sums[head]);
            int tmp = head;
            head = next[head];
            next[tmp] = -1;
            sums[tmp] = 0;
        }
        C->rowptr[i + 1] = C->nnz;
    }
    free(next);
    free(sums);
    return C;
}

/* spgemm_T_helper, matmult.cpp:139-204: C = P^T B with P's columns walked
 * in increasing row order (the CSC that CSR_to_CSC builds). */
oc_csr* oc_spgemm_T(const oc_csr* P, const oc_csr* B) {
    oc_csr* Pt = oc_csr_transpose(P);
    oc_csr* C = oc_spgemm(Pt, B);
    oc_csr_free(Pt);
    return C;
}

/* ParCSRMatrix::mult -> mult_helper -> add_append (par_matmult.cpp:73-107,
 * 244-366; add.cpp:39-78), then mult_T -> mult_T_combine -> add_append
 * (par_matmult.cpp:141-196, 387-570), then sort + move_diag
 * (par_ruge_stuben_solver.hpp:142-143) when sort_diag_first is set. */
oc_csr* oc_rap(const oc_csr* A, const oc_csr* P, int sort_diag_first) {
    oc_csr* AP = oc_spgemm(A, P);
    oc_csr_sort(AP);
    csr_remove_duplicates(AP);
    oc_csr* Ac = oc_spgemm_T(P, AP);
    oc_csr_sort(Ac);
    csr_remove_duplicates(Ac);
    if (sort_diag_first) oc_csr_move_diag(Ac);
    oc_csr_free(AP);
    return Ac;
}

/* ------------------------------------------------------------------------ */
/* smoothed aggregation (aggregation/par_*.cpp)                             */
/* ------------------------------------------------------------------------ */

#define OC_TMPSELECTION 4

/* mis2, aggregation/par_mis.cpp:204-645 (off-process parts empty) */
void oc_mis2(const oc_csr* A, const double* r, int* states) {
    int n = A->n_rows;
    int* V = (int*)malloc(sizeof(int) * (n + 1));
    int* C = (int*)calloc((size_t)n + 1, sizeof(int));
    int* next = (int*)malloc(sizeof(int) * (n + 1));
    double* row_max = (double*)malloc(sizeof(double) * (n + 1));
    for (int i = 0; i < n; i++) { V[i] = i; states[i] = OC_UNASSIGNED; next[i] = OC_UNASSIGNED; }
    /* D: directed graph, edge i->col when r[i] > r[col] */
    int* dp = (int*)calloc((size_t)n + 1, sizeof(int));
    int* di = (int*)malloc(sizeof(int) * (A->nnz + 1));
    int nd = 0;
    for (int i = 0; i < n; i++) {
        for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++)
            if (r[i] > r[A->cols[j]]) di[nd++] = A->cols[j];
        dp[i + 1] = nd;
    }
    oc_csr* At = oc_csr_transpose(A);
    int rem = n, first_pass = 1;
    while (rem || first_pass) {
        for (int t = 0; t < rem; t++) {
            int v = V[t], found = 0;
            for (int j = dp[v]; j < dp[v + 1]; j++) {
                int w = di[j];
                if (states[w] == OC_UNASSIGNED || states[w] > OC_SELECTED) { found = 1; break; }
            }
            if (!found) states[v] = OC_TMPSELECTION;
        }
        for (int i = 0; i < n; i++) {
            double mv = -1.0;
            for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) {
                int u = A->cols[j];
                if (states[u] > OC_SELECTED && r[u] > mv) mv = r[u];
            }
            row_max[i] = mv;
        }
        for (int t = 0; t < rem; t++) {
            int v = V[t], found = 0;
            if (states[v] != OC_TMPSELECTION) continue;
            for (int j = A->rowptr[v]; j < A->rowptr[v + 1]; j++)
                if (row_max[A->cols[j]] > r[v]) { found = 1; break; }
            if (!found) states[v] = OC_NEWSELECTION;
        }
        int head = OC_TMPSELECTION, length = 0;
        for (int t = 0; t < rem; t++) {
            int v = V[t];
            if (states[v] == OC_NEWSELECTION) {
                for (int j = At->rowptr[v]; j < At->rowptr[v + 1]; j++) {
                    int w = At->cols[j];
                    C[w] = OC_SELECTED;
                    if (next[w] == OC_UNASSIGNED) { next[w] = head; head = w; length++; }
                }
            }
        }
        for (int t = 0; t < rem; t++) {
            int v = V[t], found = 0;
            if (states[v] == OC_NEWSELECTION) continue;
            for (int j = A->rowptr[v]; j < A->rowptr[v + 1]; j++) {
                int w = A->cols[j];
                if (states[w] == OC_NEWSELECTION || C[w] == OC_SELECTED) { found = 1; break; }
            }
            if (found) states[v] = OC_NEWUNSELECTION;
        }
        for (int t = 0; t < length; t++) {
            int tmp = head;
            head = next[head];
            C[tmp] = OC_UNSELECTED;
            next[tmp] = 0;
        }
        int k = 0;
        for (int t = 0; t < rem; t++) {
            int v = V[t];
            if (states[v] == OC_NEWSELECTION) states[v] = OC_SELECTED;
            else if (states[v] == OC_NEWUNSELECTION) states[v] = OC_UNSELECTED;
            else V[k++] = v;
        }
        rem = k;
        first_pass = 0;
    }
    free(V); free(C); free(next); free(row_max); free(dp); free(di);
    oc_csr_free(At);
}

/* aggregate, aggregation/par_aggregate.cpp:5-185.  The SA solver passes no
 * rand_vals (r = NULL, i.e. 0); the reference test passes the weights.
 * S and A sorted with the diagonal first. */
int oc_aggregate(const oc_csr* A, const oc_csr* S, int* states, int* agg, const double* r) {
    int n = S->n_rows, n_aggs = 0;
    for (int i = 0; i < n; i++) {
        agg[i] = -1;
        if (S->rowptr[i + 1] - S->rowptr[i] <= 1) agg[i] = -n;
        else if (states[i] == OC_SELECTED) { agg[i] = i; n_aggs++; }
    }
    for (int i = 0; i < n; i++) {
        if (states[i] == OC_SELECTED) continue;
        for (int j = S->rowptr[i]; j < S->rowptr[i + 1]; j++) {
            int c = S->cols[j];
            if (states[c] == OC_SELECTED && agg[c] >= 0) { agg[i] = agg[c]; break; }
        }
    }
    for (int i = 0; i < n; i++) {
        if (agg[i] == -1) {
            int ctr = A->rowptr[i];
            double max_val = 0.0;
            int max_agg = -n;
            for (int j = S->rowptr[i]; j < S->rowptr[i + 1]; j++) {
                int c = S->cols[j];
                while (A->cols[ctr] != c) ctr++;
                double v = fabs(A->vals[ctr]) + (r ? r[c] : 0.0);
                if (v > max_val && agg[c] >= 0) { max_val = v; max_agg = agg[c]; }
            }
            agg[i] = -(max_agg + 1);
        }
    }
    for (int i = 0; i < n; i++) {
        if (agg[i] <= -n) agg[i] = -1;
        else if (agg[i] < 0) agg[i] = -(agg[i] + 1);
    }
    return n_aggs;
}

/* fit_candidates with one candidate, aggregation/par_candidates.cpp:6-216.
 * Columns of T are the used aggregate roots in increasing order. */
oc_csr* oc_fit_candidates(int n, int n_aggs, const int* agg, const double* B,
                          double* R, double tol) {
    (void)tol;
    int* used = (int*)calloc((size_t)n + 1, sizeof(int));
    for (int i = 0; i < n; i++) if (agg[i] >= 0) used[agg[i]] = 1;
    int nc = 0;
    for (int i = 0; i < n; i++) if (used[i]) used[i] = nc++ + 1;
    oc_csr* T = csr_alloc(n, n_aggs, n);
    for (int a = 0; a < n_aggs; a++) R[a] = 0.0;
    for (int i = 0; i < n; i++) {
        if (agg[i] >= 0) {
            int c = used[agg[i]] - 1;
            csr_push(T, c, B[i]);
        }
        T->rowptr[i + 1] = T->nnz;
    }
    /* R[a] accumulates over the aggregate's rows in increasing order */
    for (int i = 0; i < n; i++)
        for (int j = T->rowptr[i]; j < T->rowptr[i + 1]; j++) R[T->cols[j]] += T->vals[j] * T->vals[j];
    for (int a = 0; a < n_aggs; a++) R[a] = sqrt(R[a]);
    for (int j = 0; j < T->nnz; j++) T->vals[j] *= 1.0 / R[T->cols[j]];
    free(used);
    return T;
}

/* jacobi_prolongation, aggregation/par_prolongation.cpp:7-104 followed by
 * ParCSRMatrix::subtract (util/linalg/par_add.cpp:184-309). */
oc_csr* oc_jacobi_prolongation(const oc_csr* A, const oc_csr* T, double omega, int steps) {
    oc_csr* sA = oc_csr_copy(A);
    for (int i = 0; i < A->n_rows; i++) {
        double row_sum = 0.0, inv = 0.0;
        for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) row_sum += fabs(A->vals[j]);
        if (row_sum != 0.0) inv = (1.0 / fabs(row_sum)) * omega;
        for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) sA->vals[j] *= inv;
    }
    oc_csr* P = oc_csr_copy(T);
    for (int s = 0; s < steps; s++) {
        oc_csr* AP = oc_spgemm(sA, P);
        oc_csr_sort(AP);
        csr_remove_duplicates(AP);
        oc_csr* C = csr_alloc(P->n_rows, P->n_cols, P->nnz + AP->nnz);
        for (int i = 0; i < P->n_rows; i++) {
            for (int j = P->rowptr[i]; j < P->rowptr[i + 1]; j++) csr_push(C, P->cols[j], P->vals[j]);
            for (int j = AP->rowptr[i]; j < AP->rowptr[i + 1]; j++) csr_push(C, AP->cols[j], -AP->vals[j]);
            C->rowptr[i + 1] = C->nnz;
        }
        oc_csr_sort(C);
        csr_remove_duplicates(C);
        oc_csr_move_diag(C);
        oc_csr_free(AP);
        oc_csr_free(P);
        P = C;
    }
    oc_csr_free(sA);
    return P;
}

/* ------------------------------------------------------------------------ */
/* multicolour ordering for the multicolour SOR stand-in (not in the        */
/* reference): Jones-Plassmann rounds on the row graph of A with a fixed    */
/* integer hash as priority, ties broken by row index.  Each round colours  */
/* the uncoloured rows that beat every uncoloured neighbour with the        */
/* smallest colour unused by coloured neighbours, so the result does not    */
/* depend on the order rows are visited.                                     */
/* ------------------------------------------------------------------------ */

static uint32_t jp_hash(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
    return x;
}

static int jp_beats(int i, int j) {
    uint32_t hi = jp_hash((uint32_t)i), hj = jp_hash((uint32_t)j);
    return hi > hj || (hi == hj && i > j);
}

int oc_colour_rows(const oc_csr* A, int* colour) {
    int n = A->n_rows, left = n, ncol = 0;
    int* newc = (int*)malloc(sizeof(int) * (n + 1));
    for (int i = 0; i < n; i++) colour[i] = -1;
    while (left) {
        int nn = 0;
        for (int i = 0; i < n; i++) {
            if (colour[i] >= 0) continue;
            int ok = 1;
            for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) {
                int c = A->cols[j];
                if (c != i && colour[c] < 0 && jp_beats(c, i)) { ok = 0; break; }
            }
            if (ok) newc[nn++] = i;
        }
        for (int t = 0; t < nn; t++) {
            int i = newc[t];
            uint64_t used = 0; /* colours 0..63 */
            int c_ = 0;
            for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) {
                int c = A->cols[j];
                if (c != i && colour[c] >= 0 && colour[c] < 64) used |= (1ULL << colour[c]);
            }
            while (c_ < 64 && (used >> c_) & 1ULL) c_++;
            colour[i] = c_ + 1000; /* pending: not visible to this round */
        }
        for (int t = 0; t < nn; t++) {
            int i = newc[t];
            colour[i] -= 1000;
            if (colour[i] + 1 > ncol) ncol = colour[i] + 1;
        }
        left -= nn;
    }
    free(newc);
    return ncol;
}

/* ------------------------------------------------------------------------ */
/* relaxation (util/linalg/par_relax.cpp)                                   */
/* ------------------------------------------------------------------------ */

/* SOR_forward, par_relax.cpp:29-68 (including the row that lacks a leading
 * diagonal leaving start_on in place). */
static void sor_forward(const oc_csr* A, double* x, const double* y, double omega) {
    int start_on = 0;
    for (int i = 0; i < A->n_rows; i++) {
        double row_sum = 0, diag;
        int end_on = A->rowptr[i + 1];
        if (A->cols[start_on] == i) { diag = A->vals[start_on]; start_on++; }
        else continue;
        for (int j = start_on; j < end_on; j++) row_sum += A->vals[j] * x[A->cols[j]];
        start_on = end_on;
        x[i] = (x[i] + omega * (y[i] - x[i] - row_sum)) / diag;
    }
}

/* SOR_backward, par_relax.cpp:70-104 */
static void sor_backward(const oc_csr* A, double* x, const double* y, double omega) {
    for (int i = A->n_rows - 1; i >= 0; i--) {
        double row_sum = 0, diag;
        int s = A->rowptr[i], e = A->rowptr[i + 1];
        if (A->cols[s] == i) { diag = A->vals[s]; s++; }
        else continue;
        for (int j = s; j < e; j++) row_sum += A->vals[j] * x[A->cols[j]];
        x[i] = ((1.0 - omega) * x[i]) + (omega * ((y[i] - row_sum) / diag));
    }
}

/* jacobi_helper, par_relax.cpp:106-152.  compat=1 restates it exactly (diag
 * stays 0, so x is never written); compat=0 reads the leading diagonal. */
static void jacobi_sweep(const oc_csr* A, double* x, const double* b, double* tmp,
                         double omega, int compat) {
    int n = A->n_rows;
    OC_ROWS_PARALLEL
    for (int i = 0; i < n; i++) tmp[i] = x[i];
    OC_ROWS_PARALLEL
    for (int i = 0; i < n; i++) {
        double diag = compat ? 0.0 : A->vals[A->rowptr[i]];
        double row_sum = 0;
        for (int j = A->rowptr[i] + 1; j < A->rowptr[i + 1]; j++) row_sum += A->vals[j] * tmp[A->cols[j]];
        if (fabs(diag) > ZERO_TOL) x[i] = ((1.0 - omega) * tmp[i]) + (omega * ((b[i] - row_sum) / diag));
    }
}

/* L1-Jacobi (not in the reference): x += w (b - A x) / d_i with
 * d_i = sum_j |a_ij|, the row's l1 norm. */
static void l1_jacobi_sweep(const oc_csr* A, const double* l1, double* x, const double* b,
                            double* tmp, double omega) {
    int n = A->n_rows;
    OC_ROWS_PARALLEL
    for (int i = 0; i < n; i++) tmp[i] = x[i];
    OC_ROWS_PARALLEL
    for (int i = 0; i < n; i++) {
        double r = b[i];
        for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) r -= A->vals[j] * tmp[A->cols[j]];
        x[i] = tmp[i] + omega * r / l1[i];
    }
}

/* Multicolour forward sweep: the SOR_forward update applied colour by
 * colour; rows of one colour are uncoupled, so their order is immaterial. */
static void mc_sor_forward(const oc_csr* A, const int* colour, int ncol, double* x,
                           const double* y, double omega) {
    for (int c = 0; c < ncol; c++) {
        for (int i = 0; i < A->n_rows; i++) {
            if (colour[i] != c) continue;
            int s = A->rowptr[i], e = A->rowptr[i + 1];
            if (s == e || A->cols[s] != i) continue;
            double diag = A->vals[s], row_sum = 0;
            for (int j = s + 1; j < e; j++) row_sum += A->vals[j] * x[A->cols[j]];
            x[i] = (x[i] + omega * (y[i] - x[i] - row_sum)) / diag;
        }
    }
}

static void mc_sor_backward(const oc_csr* A, const int* colour, int ncol, double* x,
                            const double* y, double omega) {
    for (int c = ncol - 1; c >= 0; c--) {
        for (int i = 0; i < A->n_rows; i++) {
            if (colour[i] != c) continue;
            int s = A->rowptr[i], e = A->rowptr[i + 1];
            if (s == e || A->cols[s] != i) continue;
            double diag = A->vals[s], row_sum = 0;
            for (int j = s + 1; j < e; j++) row_sum += A->vals[j] * x[A->cols[j]];
            x[i] = ((1.0 - omega) * x[i]) + (omega * ((y[i] - row_sum) / diag));
        }
    }
}

static void relax(oc_ml* ml, int l, double* x, const double* b) {
    oc_level* L = &ml->lv[l];
    for (int s = 0; s < ml->o.num_smooth_sweeps; s++) {
        switch (ml->o.relax) {
        case OC_RELAX_JACOBI:
            jacobi_sweep(L->A, x, b, L->tmp, ml->o.relax_weight, ml->o.jacobi_compat);
            break;
        case OC_RELAX_SOR:
            sor_forward(L->A, x, b, ml->o.relax_weight);
            break;
        case OC_RELAX_SSOR:
            sor_forward(L->A, x, b, ml->o.relax_weight);
            sor_backward(L->A, x, b, ml->o.relax_weight);
            break;
        case OC_RELAX_L1JACOBI:
            l1_jacobi_sweep(L->A, L->l1, x, b, L->tmp, ml->o.relax_weight);
            break;
        case OC_RELAX_MCSOR:
            mc_sor_forward(L->A, L->colour, L->n_colours, x, b, ml->o.relax_weight);
            break;
        case OC_RELAX_MCSSOR:
            mc_sor_forward(L->A, L->colour, L->n_colours, x, b, ml->o.relax_weight);
            mc_sor_backward(L->A, L->colour, L->n_colours, x, b, ml->o.relax_weight);
            break;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* dense coarse solve: dgetrf_/dgetrs_ semantics (column-major, partial     */
/* pivoting on the first largest |entry|), par_multilevel.hpp:229-374       */
/* ------------------------------------------------------------------------ */

void oc_dense_lu(int n, double* a, int* piv) {
    for (int k = 0; k < n; k++) {
        int p = k;
        double mx = fabs(a[k + (size_t)k * n]);
        for (int i = k + 1; i < n; i++)
            if (fabs(a[i + (size_t)k * n]) > mx) { mx = fabs(a[i + (size_t)k * n]); p = i; }
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; j++) {
                double t = a[k + (size_t)j * n];
                a[k + (size_t)j * n] = a[p + (size_t)j * n];
                a[p + (size_t)j * n] = t;
            }
        double d = a[k + (size_t)k * n];
        if (d != 0.0)
            for (int i = k + 1; i < n; i++) a[i + (size_t)k * n] /= d;
        for (int j = k + 1; j < n; j++) {
            double akj = a[k + (size_t)j * n];
            for (int i = k + 1; i < n; i++) a[i + (size_t)j * n] -= a[i + (size_t)k * n] * akj;
        }
    }
}

void oc_dense_lu_solve(int n, const double* lu, const int* piv, double* b) {
    for (int k = 0; k < n; k++) {
        int p = piv[k];
        if (p != k) { double t = b[k]; b[k] = b[p]; b[p] = t; }
    }
    for (int j = 0; j < n; j++)
        for (int i = j + 1; i < n; i++) b[i] -= lu[i + (size_t)j * n] * b[j];
    for (int j = n - 1; j >= 0; j--) {
        b[j] /= lu[j + (size_t)j * n];
        for (int i = 0; i < j; i++) b[i] -= lu[i + (size_t)j * n] * b[j];
    }
}

/* ------------------------------------------------------------------------ */
/* hierarchy                                                                */
/* ------------------------------------------------------------------------ */

void oc_default_opts(oc_opts* o) {
    memset(o, 0, sizeof(*o));
    o->solver = OC_SOLVER_RS;
    o->interp = OC_INTERP_MODCLASSICAL;
    o->relax = OC_RELAX_JACOBI;
    o->jacobi_compat = 0;
    o->num_smooth_sweeps = 1;
    o->max_coarse = 50;
    o->max_levels = 25;
    o->max_iterations = 100;
    o->strong_threshold = 0.25;
    o->relax_weight = 1.0;
    o->solve_tol = 1e-7;
    o->interp_filter = 0.3;
    o->prolong_weight = 4.0 / 3.0;
    o->prolong_smooth_steps = 1;
}

/* form_rand_weights, par_multilevel.hpp:215-225 (glibc rand()) */
void oc_form_rand_weights(int n, int first_row, double* w) {
    srand(2448422 + first_row);
    for (int i = 0; i < n; i++) w[i] = (double)rand() / RAND_MAX;
}

static void level_alloc(oc_level* L, oc_csr* A) {
    L->A = A;
    L->n = A->n_rows;
    L->x = (double*)calloc((size_t)L->n + 1, sizeof(double));
    L->b = (double*)calloc((size_t)L->n + 1, sizeof(double));
    L->tmp = (double*)calloc((size_t)L->n + 1, sizeof(double));
}

/* ParMultilevel::setup_helper (par_multilevel.hpp:126-212) with
 * ParRugeStubenSolver::extend_hierarchy (par_ruge_stuben_solver.hpp:57-162)
 * or ParSmoothedAggregationSolver::extend_hierarchy
 * (par_smoothed_aggregation_solver.hpp:51-129), then duplicate_coarse. */
oc_ml* oc_ml_setup(const oc_csr* Af, const oc_opts* o, const double* weights, int n_weights) {
    oc_ml* ml = (oc_ml*)calloc(1, sizeof(oc_ml));
    ml->o = *o;
    oc_csr* A0 = oc_csr_copy(Af);
    oc_csr_sort(A0);
    oc_csr_move_diag(A0);
    level_alloc(&ml->lv[0], A0);
    double* w = (double*)malloc(sizeof(double) * ((size_t)Af->n_rows + 1));
    if (weights && n_weights >= Af->n_rows) memcpy(w, weights, sizeof(double) * Af->n_rows);
    else oc_form_rand_weights(Af->n_rows, o->seed_offset, w);
    double* Bc = NULL;
    if (o->solver == OC_SOLVER_SA) {
        Bc = (double*)malloc(sizeof(double) * ((size_t)Af->n_rows + 1));
        for (int i = 0; i < Af->n_rows; i++) Bc[i] = 1.0;
    }
    int nl = 1;
    while (ml->lv[nl - 1].A->n_rows > o->max_coarse && (o->max_levels == -1 || nl < o->max_levels)) {
        oc_csr* A = ml->lv[nl - 1].A;
        int n = A->n_rows;
        int* states = (int*)malloc(sizeof(int) * (n + 1));
        oc_csr* P;
        oc_csr* Ac;
        if (o->solver == OC_SOLVER_RS) {
            oc_csr* S = oc_classical_strength(A, o->strong_threshold);
            oc_split_pmis(S, w, states);
            if (o->interp == OC_INTERP_EXTENDED) P = oc_extended_interp(A, S, states, o->interp_filter);
            else if (o->interp == OC_INTERP_DIRECT) P = oc_direct_interp(A, S, states);
            else P = oc_mod_classical_interp(A, S, states);
            Ac = oc_rap(A, P, 1);
            oc_csr_free(S);
        } else {
            oc_csr_sort(A);
            oc_csr_move_diag(A);
            oc_csr* S = oc_symmetric_strength(A, o->strong_threshold);
            oc_mis2(S, w, states);
            int* agg = (int*)malloc(sizeof(int) * (n + 1));
            int n_aggs = oc_aggregate(A, S, states, agg, NULL);
            double* R = (double*)malloc(sizeof(double) * ((size_t)n_aggs + 1));
            oc_csr* T = oc_fit_candidates(n, n_aggs, agg, Bc, R, 1e-10);
            P = oc_jacobi_prolongation(A, T, o->prolong_weight, o->prolong_smooth_steps);
            Ac = oc_rap(A, P, 0);
            for (int a = 0; a < n_aggs; a++) Bc[a] = R[a];
            oc_csr_free(T);
            free(agg);
            free(R);
            oc_csr_free(S);
        }
        ml->lv[nl - 1].P = P;
        level_alloc(&ml->lv[nl], Ac);
        free(states);
        nl++;
    }
    ml->num_levels = nl;
    /* relaxation needs diagonal-first rows on every smoothed level
     * (par_relax.cpp:157-159 sorts lazily) */
    for (int l = 0; l < nl; l++) {
        oc_csr_sort(ml->lv[l].A);
        oc_csr_move_diag(ml->lv[l].A);
    }
    for (int l = 0; l < nl - 1; l++) {
        oc_level* L = &ml->lv[l];
        L->l1 = (double*)calloc((size_t)L->n + 1, sizeof(double));
        for (int i = 0; i < L->n; i++) {
            double s = 0;
            for (int j = L->A->rowptr[i]; j < L->A->rowptr[i + 1]; j++) s += fabs(L->A->vals[j]);
            L->l1[i] = s;
        }
        L->colour = (int*)malloc(sizeof(int) * ((size_t)L->n + 1));
        L->n_colours = oc_colour_rows(L->A, L->colour);
    }
    /* duplicate_coarse: row-major dense A_c handed to column-major dgetrf */
    oc_csr* Ac = ml->lv[nl - 1].A;
    int cn = Ac->n_rows;
    ml->coarse_n = cn;
    ml->lu = (double*)calloc((size_t)cn * cn + 1, sizeof(double));
    ml->piv = (int*)calloc((size_t)cn + 1, sizeof(int));
    for (int i = 0; i < cn; i++)
        for (int j = Ac->rowptr[i]; j < Ac->rowptr[i + 1]; j++) ml->lu[(size_t)i * cn + Ac->cols[j]] = Ac->vals[j];
    oc_dense_lu(cn, ml->lu, ml->piv);
    free(w);
    free(Bc);
    return ml;
}

void oc_ml_free(oc_ml* ml) {
    if (!ml) return;
    for (int l = 0; l < ml->num_levels; l++) {
        oc_level* L = &ml->lv[l];
        oc_csr_free(L->A);
        oc_csr_free(L->P);
        free(L->x); free(L->b); free(L->tmp); free(L->colour); free(L->l1);
    }
    free(ml->lu);
    free(ml->piv);
    free(ml);
}

int oc_ml_num_levels(const oc_ml* ml) { return ml->num_levels; }
const oc_csr* oc_ml_level_A(const oc_ml* ml, int l) { return ml->lv[l].A; }
const oc_csr* oc_ml_level_P(const oc_ml* ml, int l) { return ml->lv[l].P; }

/* ParMultilevel::cycle, par_multilevel.hpp:341-457 */
static void cycle(oc_ml* ml, double* x, const double* b, int l) {
    oc_level* L = &ml->lv[l];
    if (l == ml->num_levels - 1) {
        double* bd = (double*)malloc(sizeof(double) * ((size_t)ml->coarse_n + 1));
        memcpy(bd, b, sizeof(double) * ml->coarse_n);
        oc_dense_lu_solve(ml->coarse_n, ml->lu, ml->piv, bd);
        memcpy(x, bd, sizeof(double) * ml->coarse_n);
        free(bd);
        return;
    }
    oc_level* C = &ml->lv[l + 1];
    memset(C->x, 0, sizeof(double) * C->n);
    relax(ml, l, x, b);
    oc_residual(L->A, x, b, L->tmp);
    oc_spmv_T(L->P, L->tmp, C->b);
    cycle(ml, C->x, C->b, l + 1);
    oc_spmv_append(L->P, C->x, x);
    relax(ml, l, x, b);
}

void oc_ml_cycle(oc_ml* ml, double* x, const double* b) { cycle(ml, x, b, 0); }

/* Vector::norm, vector.cpp:107-118, and ParVector::norm, par_vector.cpp:88-98 */
static double vnorm(const double* v, int n) {
    double r = 0.0;
    for (int i = 0; i < n; i++)
        if (fabs(v[i]) > ZERO_TOL) r += pow(v[i], 2);
    r = pow(r, 1.0 / 2);
    r = pow(r, 2);
    return pow(r, 1. / 2);
}

static double vdot(const double* a, const double* b, int n) {
    double r = 0.0;
    for (int i = 0; i < n; i++) r += a[i] * b[i];
    return r;
}

static void vaxpy(double* y, const double* x, double a, int n) {
    OC_ROWS_PARALLEL
    for (int i = 0; i < n; i++) y[i] += x[i] * a;
}

/* ParMultilevel::solve, par_multilevel.hpp:459-538 */
int oc_ml_solve(oc_ml* ml, double* x, const double* b, double* hist, int cap) {
    int n = ml->lv[0].n, iter = 0;
    double b_norm = vnorm(b, n), r_norm;
    double* r = (double*)malloc(sizeof(double) * ((size_t)n + 1));
    oc_residual(ml->lv[0].A, x, b, r);
    r_norm = fabs(b_norm) > ZERO_TOL ? vnorm(r, n) / b_norm : vnorm(r, n);
    if (cap > 0) hist[0] = r_norm;
    while (r_norm > ml->o.solve_tol && iter < ml->o.max_iterations) {
        cycle(ml, x, b, 0);
        iter++;
        oc_residual(ml->lv[0].A, x, b, r);
        r_norm = fabs(b_norm) > ZERO_TOL ? vnorm(r, n) / b_norm : vnorm(r, n);
        if (iter < cap) hist[iter] = r_norm;
    }
    free(r);
    return iter;
}

/* PCG, krylov/par_cg.cpp:121-263.  Returns the number of history entries
 * (res[0] = sqrt(r.z), then r.z / b.Mb per iteration); stops on
 * next_inner < tol*sqrt(b.Mb); restarts every 8 iterations. */
int oc_pcg_mode(const oc_csr* A, oc_ml* ml, double* x, const double* b, double tol,
                int max_iter, int mode, double* hist, int cap);

int oc_pcg(const oc_csr* A, oc_ml* ml, double* x, const double* b, double tol, int max_iter,
           double* hist, int cap) {
    return oc_pcg_mode(A, ml, x, b, tol, max_iter, 0, hist, cap);
}

/* mode 0: the reference's iteration exactly.  mode 1 (not in the reference):
 * the same recurrence stopped when ||r|| <= tol ||b|| with the true residual
 * confirmed at exit, residual replacement every 10 iterations and no p
 * restart; history entries ||r||/||b||. */
int oc_pcg_mode(const oc_csr* A, oc_ml* ml, double* x, const double* b, double tol,
                int max_iter, int mode, double* hist, int cap) {
    int n = A->n_rows;
    if (max_iter <= 0) max_iter = (int)(1.3 * n) + 2;
    double* r = (double*)calloc((size_t)n + 1, sizeof(double));
    double* z = (double*)calloc((size_t)n + 1, sizeof(double));
    double* p = (double*)calloc((size_t)n + 1, sizeof(double));
    double* Ap = (double*)calloc((size_t)n + 1, sizeof(double));
    int nh = 0;
    if (mode == 1) {
        double bn = sqrt(vdot(b, b, n));
        if (bn == 0.0) bn = 1.0;
        oc_residual(A, x, b, r);
        memset(z, 0, sizeof(double) * n);
        cycle(ml, z, r, 0);
        memcpy(p, z, sizeof(double) * n);
        double rz = vdot(r, z, n);
        double rn = sqrt(vdot(r, r, n));
        if (nh < cap) hist[nh] = rn / bn;
        nh++;
        int it = 0;
        while (rn > tol * bn && it < max_iter) {
            it++;
            oc_spmv(A, p, Ap);
            double pAp = vdot(Ap, p, n);
            double alpha = rz / pAp;
            vaxpy(x, p, alpha, n);
            if (it % 10 == 0) oc_residual(A, x, b, r);
            else vaxpy(r, Ap, -alpha, n);
            rn = sqrt(vdot(r, r, n));
            if (rn <= tol * bn) {
                oc_residual(A, x, b, r);
                rn = sqrt(vdot(r, r, n));
            }
            if (nh < cap) hist[nh] = rn / bn;
            nh++;
            if (rn <= tol * bn) break;
            memset(z, 0, sizeof(double) * n);
            cycle(ml, z, r, 0);
            double next = vdot(r, z, n);
            double beta = next / rz;
            OC_ROWS_PARALLEL
            for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
            rz = next;
        }
        free(r); free(z); free(p); free(Ap);
        return nh;
    }
    memset(z, 0, sizeof(double) * n);
    cycle(ml, z, b, 0);
    double b_inner = vdot(b, z, n);
    double norm_b = sqrt(b_inner);
    if (norm_b > ZERO_TOL) tol = tol * norm_b;
    oc_residual(A, x, b, r);
    memset(z, 0, sizeof(double) * n);
    cycle(ml, z, r, 0);
    memcpy(p, z, sizeof(double) * n);
    double rz = vdot(r, z, n);
    if (nh < cap) hist[nh] = sqrt(rz);
    nh++;
    int iter = 0;
    while (iter < max_iter) {
        iter++;
        oc_spmv(A, p, Ap);
        double pAp = vdot(Ap, p, n);
        if (pAp < 0.0) { nh = -nh; break; }
        double alpha = rz / pAp;
        vaxpy(x, p, alpha, n);
        int full_r = iter % 8 == 0;
        if (full_r) oc_residual(A, x, b, r);
        else vaxpy(r, Ap, -1.0 * alpha, n);
        memset(z, 0, sizeof(double) * n);
        cycle(ml, z, r, 0);
        double next = vdot(r, z, n);
        double beta = next / rz;
        if (nh < cap) hist[nh] = next / b_inner;
        nh++;
        if (next < tol) break;
        if (full_r) memcpy(p, z, sizeof(double) * n);
        else {
            for (int i = 0; i < n; i++) p[i] *= beta;
            vaxpy(p, z, 1.0, n);
        }
        rz = next;
    }
    free(r); free(z); free(p); free(Ap);
    return nh;
}

/* CG, krylov/par_cg.cpp:8-118; history entries are ||r||/||b||. */
int oc_cg(const oc_csr* A, double* x, const double* b, double tol, int max_iter, double* hist,
          int cap) {
    int n = A->n_rows;
    double b_norm = vnorm(b, n);
    if (b_norm < ZERO_TOL) b_norm = 1.0;
    if (max_iter <= 0) max_iter = (int)(1.3 * n) + 2;
    double* r = (double*)calloc((size_t)n + 1, sizeof(double));
    double* p = (double*)calloc((size_t)n + 1, sizeof(double));
    double* Ap = (double*)calloc((size_t)n + 1, sizeof(double));
    oc_residual(A, x, b, r);
    memcpy(p, r, sizeof(double) * n);
    double rr = vdot(r, r, n);
    double norm_r = sqrt(rr);
    int nh = 0;
    if (nh < cap) hist[nh] = norm_r / b_norm;
    nh++;
    if (norm_r != 0.0) tol = tol * norm_r;
    int iter = 0;
    while (norm_r > tol && iter < max_iter) {
        oc_spmv(A, p, Ap);
        double pAp = vdot(Ap, p, n);
        if (pAp < 0.0) { nh = -nh; break; }
        double alpha = rr / pAp;
        vaxpy(x, p, alpha, n);
        if ((iter % 8) && iter > 0) vaxpy(r, Ap, -1.0 * alpha, n);
        else oc_residual(A, x, b, r);
        double next = vdot(r, r, n);
        double beta = next / rr;
        for (int i = 0; i < n; i++) p[i] *= beta;
        vaxpy(p, r, 1.0, n);
        rr = next;
        norm_r = sqrt(rr);
        if (nh < cap) hist[nh] = norm_r / b_norm;
        nh++;
        iter++;
    }
    free(r); free(p); free(Ap);
    return nh;
}

/* BiCGStab, krylov/par_bicgstab.cpp:11-126 (ml == NULL) and Pre_BiCGStab,
 * :240-371 with its uninitialised iteration counter set to 0 and the
 * preconditioned vectors sized; history entries are ||r||. */
static int bicgstab_impl(const oc_csr* A, oc_ml* ml, double* x, const double* b, double tol,
                         int max_iter, double* hist, int cap) {
    int n = A->n_rows;
    if (max_iter <= 0) max_iter = (int)(1.3 * n) + 2;
    double* r = (double*)calloc((size_t)n + 1, sizeof(double));
    double* rs = (double*)calloc((size_t)n + 1, sizeof(double));
    double* s = (double*)calloc((size_t)n + 1, sizeof(double));
    double* p = (double*)calloc((size_t)n + 1, sizeof(double));
    double* Ap = (double*)calloc((size_t)n + 1, sizeof(double));
    double* As = (double*)calloc((size_t)n + 1, sizeof(double));
    double* ph = (double*)calloc((size_t)n + 1, sizeof(double));
    double* sh = (double*)calloc((size_t)n + 1, sizeof(double));
    oc_residual(A, x, b, r);
    memcpy(rs, r, sizeof(double) * n);
    memcpy(p, r, sizeof(double) * n);
    double rr = vdot(r, rs, n);
    double norm_r = vnorm(r, n);
    int nh = 0;
    if (nh < cap) hist[nh] = norm_r;
    nh++;
    if (norm_r != 0.0) tol = tol * norm_r;
    int iter = 0;
    while (norm_r > tol && iter < max_iter) {
        const double* pv = p;
        if (ml) { memset(ph, 0, sizeof(double) * n); cycle(ml, ph, p, 0); pv = ph; }
        oc_spmv(A, pv, Ap);
        double Apr = vdot(Ap, rs, n);
        double alpha = rr / Apr;
        memcpy(s, r, sizeof(double) * n);
        vaxpy(s, Ap, -1.0 * alpha, n);
        const double* sv = s;
        if (ml) { memset(sh, 0, sizeof(double) * n); cycle(ml, sh, s, 0); sv = sh; }
        oc_spmv(A, sv, As);
        double As_s = vdot(As, s, n);
        double AsAs = vdot(As, As, n);
        double omega = As_s / AsAs;
        vaxpy(x, pv, alpha, n);
        vaxpy(x, sv, omega, n);
        memcpy(r, s, sizeof(double) * n);
        vaxpy(r, As, -1.0 * omega, n);
        double next = vdot(r, rs, n);
        double beta = (next / rr) * (alpha / omega);
        for (int i = 0; i < n; i++) p[i] *= beta;
        vaxpy(p, r, 1.0, n);
        vaxpy(p, Ap, -1.0 * beta * omega, n);
        rr = next;
        norm_r = vnorm(r, n);
        if (nh < cap) hist[nh] = norm_r;
        nh++;
        iter++;
    }
    free(r); free(rs); free(s); free(p); free(Ap); free(As); free(ph); free(sh);
    return nh;
}

int oc_bicgstab(const oc_csr* A, double* x, const double* b, double tol, int max_iter,
                double* hist, int cap) {
    return bicgstab_impl(A, NULL, x, b, tol, max_iter, hist, cap);
}

int oc_pre_bicgstab(const oc_csr* A, oc_ml* ml, double* x, const double* b, double tol,
                    int max_iter, double* hist, int cap) {
    return bicgstab_impl(A, ml, x, b, tol, max_iter, hist, cap);
}
