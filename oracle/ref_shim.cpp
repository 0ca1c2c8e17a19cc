// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-callable shim over the reference's own *sequential* routines
// (13manan/raptor, compiled unmodified from its sources by oracle/build.py
// into oracle/_ref/).  Each entry point copies plain arrays into a reference
// CSRMatrix, calls the reference routine, and hands the result back as a
// malloc'd triple that rs_free() releases.  It is used only to cross-check the
// C restatement in raptor_oracle.c on inputs larger than the golden fixtures.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "core/matrix.hpp"
#include "core/types.hpp"
#include "aggregation/aggregate.hpp"
#include "aggregation/mis.hpp"
#include "ruge_stuben/cf_splitting.hpp"
#include "ruge_stuben/interpolation.hpp"

using namespace raptor;

namespace {

CSRMatrix* make_csr(int n_rows, int n_cols, const int* rowptr, const int* cols,
                    const double* vals) {
    aligned_vector<int> rp(rowptr, rowptr + n_rows + 1);
    int nnz = rowptr[n_rows];
    aligned_vector<int> ci(cols, cols + nnz);
    aligned_vector<double> cv(vals, vals + nnz);
    CSRMatrix* A = new CSRMatrix(n_rows, n_cols, rp, ci, cv);
    return A;
}

struct Out {
    int n_rows, n_cols, nnz;
    int* rowptr;
    int* cols;
    double* vals;
};

Out* export_csr(CSRMatrix* A) {
    Out* o = (Out*)malloc(sizeof(Out));
    o->n_rows = A->n_rows;
    o->n_cols = A->n_cols;
    o->nnz = A->idx1[A->n_rows];
    o->rowptr = (int*)malloc(sizeof(int) * (o->n_rows + 1));
    o->cols = (int*)malloc(sizeof(int) * (o->nnz + 1));
    o->vals = (double*)malloc(sizeof(double) * (o->nnz + 1));
    memcpy(o->rowptr, A->idx1.data(), sizeof(int) * (o->n_rows + 1));
    if (o->nnz) {
        memcpy(o->cols, A->idx2.data(), sizeof(int) * o->nnz);
        memcpy(o->vals, A->vals.data(), sizeof(double) * o->nnz);
    }
    return o;
}

// A reference BSRMatrix holding block CSR arrays (block j's values at
// vals[j*br*bc], row-major).  The members are filled directly: the
// (rowptr, cols, data) constructor (core/matrix.hpp:984-993) starts from
// CSRMatrix(n, m, 0), whose n+1 zero row pointers init_from_lists then
// appends the given ones to, leaving every block row empty.
BSRMatrix* make_bsr(int nbr, int nbc, int br, int bc, const int* rp, const int* ci,
                    const double* v) {
    BSRMatrix* A = new BSRMatrix(nbr, nbc, br, bc);
    const int nnz = rp[nbr];
    std::copy(rp, rp + nbr + 1, A->idx1.begin());
    A->idx2.assign(ci, ci + nnz);
    const size_t bs = (size_t)br * bc;
    for (int j = 0; j < nnz; j++) {
        double* blk = new double[bs];
        std::copy(v + j * bs, v + (j + 1) * bs, blk);
        A->block_vals.push_back(blk);
    }
    A->nnz = nnz;
    return A;
}

}  // namespace

extern "C" {

void rs_free(Out* o) {
    if (!o) return;
    free(o->rowptr);
    free(o->cols);
    free(o->vals);
    free(o);
}

void rs_info(const Out* o, int* n_rows, int* n_cols, int* nnz) {
    *n_rows = o->n_rows;
    *n_cols = o->n_cols;
    *nnz = o->nnz;
}

void rs_export(const Out* o, int* rowptr, int* cols, double* vals) {
    memcpy(rowptr, o->rowptr, sizeof(int) * (o->n_rows + 1));
    if (o->nnz) {
        memcpy(cols, o->cols, sizeof(int) * o->nnz);
        memcpy(vals, o->vals, sizeof(double) * o->nnz);
    }
}

void rs_spmv(int n_rows, int n_cols, const int* rp, const int* ci, const double* cv,
             const double* x, double* b) {
    CSRMatrix* A = make_csr(n_rows, n_cols, rp, ci, cv);
    A->spmv(x, b);
    delete A;
}

void rs_residual(int n_rows, int n_cols, const int* rp, const int* ci, const double* cv,
                 const double* x, const double* b, double* r) {
    CSRMatrix* A = make_csr(n_rows, n_cols, rp, ci, cv);
    A->spmv_residual(x, b, r);
    delete A;
}

// C = A * B through Matrix::mult (spgemm_helper, then no add_append).
Out* rs_spgemm(int an, int am, const int* arp, const int* aci, const double* acv, int bn,
               int bm, const int* brp, const int* bci, const double* bcv) {
    CSRMatrix* A = make_csr(an, am, arp, aci, acv);
    CSRMatrix* B = make_csr(bn, bm, brp, bci, bcv);
    CSRMatrix* C = A->mult(B);
    Out* o = export_csr(C);
    delete A;
    delete B;
    delete C;
    return o;
}

// C = P^T * B through Matrix::mult_T (P converted to CSC, spgemm_T_helper).
Out* rs_spgemm_T(int pn, int pm, const int* prp, const int* pci, const double* pcv, int bn,
                 int bm, const int* brp, const int* bci, const double* bcv) {
    CSRMatrix* P = make_csr(pn, pm, prp, pci, pcv);
    CSRMatrix* B = make_csr(bn, bm, brp, bci, bcv);
    CSRMatrix* C = B->mult_T(P);
    Out* o = export_csr(C);
    delete P;
    delete B;
    delete C;
    return o;
}

Out* rs_strength(int n, const int* rp, const int* ci, const double* cv, double theta,
                 int symmetric) {
    CSRMatrix* A = make_csr(n, n, rp, ci, cv);
    CSRMatrix* S = A->strength(symmetric ? Symmetric : Classical, theta);
    Out* o = export_csr(S);
    delete A;
    delete S;
    return o;
}

void rs_split_pmis(int n, const int* rp, const int* ci, const double* cv, double* weights,
                   int* states_out) {
    CSRMatrix* S = make_csr(n, n, rp, ci, cv);
    aligned_vector<int> states;
    split_pmis(S, states, weights);
    for (int i = 0; i < n; i++) states_out[i] = states[i];
    delete S;
}

void rs_split_rs(int n, const int* rp, const int* ci, const double* cv, int second_pass,
                 int* states_out) {
    CSRMatrix* S = make_csr(n, n, rp, ci, cv);
    aligned_vector<int> states;
    split_rs(S, states, false, second_pass != 0);
    for (int i = 0; i < n; i++) states_out[i] = states[i];
    delete S;
}

void rs_split_cljp(int n, const int* rp, const int* ci, const double* cv, double* weights,
                   int* states_out) {
    CSRMatrix* S = make_csr(n, n, rp, ci, cv);
    aligned_vector<int> states;
    split_cljp(S, states, weights);
    for (int i = 0; i < n; i++) states_out[i] = states[i];
    delete S;
}

void rs_mis2(int n, const int* rp, const int* ci, const double* cv, double* weights,
             int* states_out) {
    CSRMatrix* S = make_csr(n, n, rp, ci, cv);
    aligned_vector<int> states;
    mis2(S, states, weights);
    for (int i = 0; i < n; i++) states_out[i] = states[i];
    delete S;
}

Out* rs_interp(int n, const int* arp, const int* aci, const double* acv, const int* srp,
               const int* sci, const double* scv, const int* states_in, int extended) {
    CSRMatrix* A = make_csr(n, n, arp, aci, acv);
    CSRMatrix* S = make_csr(n, n, srp, sci, scv);
    aligned_vector<int> states(states_in, states_in + n);
    // extended: 0 mod_classical, 1 extended, 2 direct
    CSRMatrix* P = extended == 1   ? extended_interpolation(A, S, states)
                   : extended == 2 ? direct_interpolation(A, S, states)
                                   : mod_classical_interpolation(A, S, states);
    Out* o = export_csr(P);
    delete A;
    delete S;
    delete P;
    return o;
}

// Block products through the reference's Matrix templates
// (core/matrix.hpp:338-368): op 0 mult (out = A x), 1 mult_append (out = b,
// then += A x), 2 residual (out = b - A x), 3 mult_T (out = A^T x).
void rs_bsr_apply(int nbr, int nbc, int br, int bc, const int* rp, const int* ci,
                  const double* v, int op, const double* x, const double* b, double* out) {
    BSRMatrix* A = make_bsr(nbr, nbc, br, bc, rp, ci, v);
    double* xp = const_cast<double*>(x);
    double* bp = const_cast<double*>(b);
    switch (op) {
        case 0: A->mult(xp, out); break;
        case 1:
            std::copy(b, b + (size_t)nbr * br, out);
            A->mult_append(xp, out);
            break;
        case 2: A->residual(xp, bp, out); break;
        case 3: A->mult_T(xp, out); break;
    }
    delete A;
}

// BSRMatrix::to_CSR (core/matrix.cpp:1180-1185).
Out* rs_bsr_to_csr(int nbr, int nbc, int br, int bc, const int* rp, const int* ci,
                   const double* v) {
    BSRMatrix* A = make_bsr(nbr, nbc, br, bc, rp, ci, v);
    CSRMatrix* C = A->to_CSR();
    Out* o = export_csr(C);
    delete C;
    delete A;
    return o;
}

// BSRMatrix::sort, move_diag, remove_duplicates (the order of the
// reference's test_block_matrix.cpp); writes the result, returns its blocks.
// The block pointers are released here, not by the destructor: dropping a
// block in remove_duplicates_helper copies pointers between slots.
int rs_bsr_sort_diag_first(int nbr, int nbc, int br, int bc, const int* rp, const int* ci,
                           const double* v, int* out_rp, int* out_ci, double* out_v) {
    BSRMatrix* A = make_bsr(nbr, nbc, br, bc, rp, ci, v);
    A->sort();
    A->move_diag();
    A->remove_duplicates();
    const size_t bs = (size_t)br * bc;
    std::copy(A->idx1.begin(), A->idx1.begin() + nbr + 1, out_rp);
    std::copy(A->idx2.begin(), A->idx2.begin() + A->nnz, out_ci);
    for (int j = 0; j < A->nnz; j++)
        std::copy(A->block_vals[j], A->block_vals[j] + bs, out_v + j * bs);
    const int nnz = A->nnz;
    A->block_vals.clear();
    delete A;
    return nnz;
}

// BCOOMatrix::add_value per block, then to_BSR (core/matrix.cpp:1116-1123):
// the block CSR arrays are written to rp (nbr+1), ci (nnz) and v (nnz*br*bc).
void rs_bcoo_to_bsr(int nbr, int nbc, int br, int bc, int nnz, const int* rows,
                    const int* cols, const double* vals, int* rp, int* ci, double* v) {
    BCOOMatrix* B = new BCOOMatrix(nbr, nbc, br, bc);
    const size_t bs = (size_t)br * bc;
    for (int k = 0; k < nnz; k++)
        B->add_value(rows[k], cols[k], const_cast<double*>(vals + k * bs));
    BSRMatrix* A = (BSRMatrix*)B->to_BSR();
    std::copy(A->idx1.begin(), A->idx1.begin() + nbr + 1, rp);
    std::copy(A->idx2.begin(), A->idx2.begin() + A->nnz, ci);
    for (int j = 0; j < A->nnz; j++) std::copy(A->block_vals[j], A->block_vals[j] + bs, v + j * bs);
    delete A;
    delete B;
}

}  // extern "C"
