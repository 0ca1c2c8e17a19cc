// aggregation.cu -- smoothed-aggregation setup kernels, FP64, bit-exact.
//
// mis2 (aggregation/par_mis.cpp:204-645), aggregate
// (aggregation/par_aggregate.cpp:5-185), fit_candidates with one candidate
// (aggregation/par_candidates.cpp:6-216) and jacobi_prolongation
// (aggregation/par_prolongation.cpp:7-104, then ParCSRMatrix::subtract) at
// world size 1.  Built with -fmad=false; products and sums spell out the
// rounding so every value matches the reference's x86-64 build bit for bit.
//
// The reference walks its node lists sequentially.  Each of its passes is
// restated here as data-parallel kernels that read a snapshot and write a
// second buffer wherever a node's new value depends on a neighbour's value
// from the same pass, so the result does not depend on thread order and
// equals the sequential one (the arguments are given at each kernel).
#include <algorithm>
#include <climits>
#include <memory>
#include <vector>

#include "rb_internal.cuh"

namespace rb {

namespace {

constexpr double kZeroTol = 1e-16;   // core/types.hpp:26
constexpr int kSelected = 1, kUnselected = 0, kUnassigned = -1;
constexpr int kNewSelection = 3, kNewUnselection = 2, kTmpSelection = 4;

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }

__device__ __forceinline__ bool remaining(int s) { return s == kUnassigned || s == kTmpSelection; }

// ================================================================= MIS2 ===
// One pass of the reference's loop (par_mis.cpp:340-640).  A node is in the
// remaining list V exactly when its state is Unassigned or TmpSelection, so
// the list is kept implicitly by the states.

// Phase 1: a remaining v with no D-neighbour w (r[v] > r[w]) that is
// Unassigned or above Selected becomes TmpSelection.  A neighbour's state
// can only move from Unassigned to TmpSelection during the pass, and both
// count, so reading the pre-pass snapshot gives the sequential answer.
__global__ void k_mis2_tmp(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ r, const int* __restrict__ st,
                           int* __restrict__ st_out) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int s = st[v];
    if (!remaining(s)) { st_out[v] = s; return; }
    const double rv = r[v];
    bool found = false;
    for (int j = rp[v]; j < rp[v + 1]; j++) {
        const int w = ci[j];
        if (rv > r[w]) {
            const int sw = st[w];
            if (sw == kUnassigned || sw > kSelected) { found = true; break; }
        }
    }
    st_out[v] = found ? s : kTmpSelection;
}

// Phase 2: the largest weight among each row's neighbours above Selected.
__global__ void k_mis2_rowmax(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                              const double* __restrict__ r, const int* __restrict__ st,
                              double* __restrict__ row_max) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double mv = -1.0;
    for (int j = rp[i]; j < rp[i + 1]; j++) {
        const int u = ci[j];
        if (st[u] > kSelected && r[u] > mv) mv = r[u];
    }
    row_max[i] = mv;
}

// Phase 3: a TmpSelection v none of whose neighbours has a larger row_max
// becomes NewSelection (row_max is fixed for the pass).
__global__ void k_mis2_select(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                              const double* __restrict__ r, const double* __restrict__ row_max,
                              int* st) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n || st[v] != kTmpSelection) return;
    const double rv = r[v];
    for (int j = rp[v]; j < rp[v + 1]; j++)
        if (row_max[ci[j]] > rv) return;
    st[v] = kNewSelection;
}

// Phase 4: the reference marks C[w] for every w whose row holds a new
// selection v (it walks S^T from v); here each w reads its own row.  The
// reference also threads each marked w onto a list and, after the pass,
// clears C[w] for the listed nodes -- but it resets a listed node's link to
// 0, not to Unassigned, so a node is listed only the first time it is
// marked; after a later marking its C stays set for the rest of the loop.
// `listed` records that, and `fresh` the nodes this pass lists.
__global__ void k_mis2_mark(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                            const int* __restrict__ st, int* C, const int* __restrict__ listed,
                            int* fresh) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n) return;
    bool m = false;
    for (int j = rp[w]; j < rp[w + 1]; j++)
        if (st[ci[j]] == kNewSelection) { m = true; break; }
    fresh[w] = (m && !listed[w]) ? 1 : 0;
    if (m) C[w] = kSelected;
}

// Phase 5: a remaining v that is not a new selection and neighbours a new
// selection or a marked node becomes NewUnselection.  Reads the snapshot st
// (NewSelection does not change in this phase), writes st_out.
__global__ void k_mis2_unselect(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                const int* __restrict__ st, const int* __restrict__ C,
                                int* __restrict__ st_out) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int s = st[v];
    st_out[v] = s;
    if (s == kNewSelection || !remaining(s)) return;
    for (int j = rp[v]; j < rp[v + 1]; j++) {
        const int w = ci[j];
        if (st[w] == kNewSelection || C[w] == kSelected) { st_out[v] = kNewUnselection; return; }
    }
}

// End of pass: clear the nodes listed this pass, commit the new states and
// count the nodes still remaining.
__global__ void k_mis2_commit(int n, int* st, int* C, int* listed, const int* __restrict__ fresh,
                              int* rem) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    if (fresh[v]) { C[v] = kUnselected; listed[v] = 1; }
    const int s = st[v];
    if (s == kNewSelection) st[v] = kSelected;
    else if (s == kNewUnselection) st[v] = kUnselected;
    else if (remaining(s)) atomicAdd(rem, 1);
}

__global__ void k_fill_int(int n, int* a, int v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

// ============================================================ aggregate ===
// par_aggregate.cpp:73-87: isolated rows (only the diagonal) get -n, roots
// their own index.
__global__ void k_agg_init(int n, const int* __restrict__ srp, const int* __restrict__ st,
                           int* agg, int* n_aggs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (srp[i + 1] - srp[i] <= 1) agg[i] = -n;
    else if (st[i] == kSelected) { agg[i] = i; atomicAdd(n_aggs, 1); }
    else agg[i] = -1;
}

// Pass 1 (:96-132): a non-root joins the first root in its row.  Only
// non-roots are written and only roots are read, so the pass is parallel.
__global__ void k_agg_pass1(int n, const int* __restrict__ srp, const int* __restrict__ sci,
                            const int* __restrict__ st, int* agg) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || st[i] == kSelected) return;
    for (int j = srp[i]; j < srp[i + 1]; j++) {
        const int c = sci[j];
        if (st[c] == kSelected && agg[c] >= 0) { agg[i] = agg[c]; return; }
    }
}

// Pass 2 (:139-186): a still unassigned row joins the aggregate of its
// strongest assigned neighbour, value |a_ic| + r_c, encoded -(agg + 1).
// The sequential loop reads values written earlier in the same loop; those
// are negative (never "assigned") except when a row found no neighbour at
// all, whose code -(-n + 1) = n - 1 is not negative.  So this parallel pass
// reads the snapshot agg_in and counts such rows; when there are none its
// result is the sequential one, and otherwise k_agg_pass2_seq runs instead.
__device__ __forceinline__ int agg_pass2_row(int i, int n, const int* __restrict__ arp,
                                             const int* __restrict__ aci,
                                             const double* __restrict__ acv,
                                             const int* __restrict__ srp,
                                             const int* __restrict__ sci,
                                             const double* __restrict__ r, const int* agg,
                                             int* bad) {
    int ctr = arp[i];
    const int aend = arp[i + 1];
    double max_val = 0.0;
    int max_agg = -n;
    for (int j = srp[i]; j < srp[i + 1]; j++) {
        const int c = sci[j];
        while (ctr < aend && aci[ctr] != c) ctr++;
        if (ctr == aend) { atomicAdd(bad, 1); break; }   // S entry missing from A's row
        const double val = dadd(fabs(acv[ctr]), r ? r[c] : 0.0);
        if (val > max_val && agg[c] >= 0) { max_val = val; max_agg = agg[c]; }
    }
    return -(max_agg + 1);
}

__global__ void k_agg_pass2(int n, const int* __restrict__ arp, const int* __restrict__ aci,
                            const double* __restrict__ acv, const int* __restrict__ srp,
                            const int* __restrict__ sci, const double* __restrict__ r,
                            const int* __restrict__ agg_in, int* __restrict__ agg_out,
                            int* none_found, int* bad) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int a = agg_in[i];
    if (a != -1) { agg_out[i] = a; return; }
    const int code = agg_pass2_row(i, n, arp, aci, acv, srp, sci, r, agg_in, bad);
    if (code == n - 1) atomicAdd(none_found, 1);
    agg_out[i] = code;
}

// The sequential pass 2, in place, for the inputs where order matters.
__global__ void k_agg_pass2_seq(int n, const int* __restrict__ arp, const int* __restrict__ aci,
                                const double* __restrict__ acv, const int* __restrict__ srp,
                                const int* __restrict__ sci, const double* __restrict__ r,
                                int* agg, int* bad) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int i = 0; i < n; i++)
        if (agg[i] == -1) agg[i] = agg_pass2_row(i, n, arp, aci, acv, srp, sci, r, agg, bad);
}

// :188-194: decode.
__global__ void k_agg_final(int n, int* agg) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int a = agg[i];
    if (a <= -n) agg[i] = -1;
    else if (a < 0) agg[i] = -(a + 1);
}

// ======================================================= fit_candidates ===
__global__ void k_mark_used(int n, const int* __restrict__ agg, int* used, int* has) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int a = agg[i];
    has[i] = a >= 0 ? 1 : 0;
    if (a >= 0 && a < n) atomicOr(used + a, 1);
}

// T row i: one entry (coarse index of its root, B_i) when aggregated.
__global__ void k_tent_fill(int n, const int* __restrict__ agg, const int* __restrict__ cidx,
                            const int* __restrict__ trp, const double* __restrict__ B, int* tci,
                            double* tcv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int a = agg[i];
    if (a < 0) return;
    tci[trp[i]] = cidx[a];
    tcv[trp[i]] = B[i];
}

// R_a = sqrt(sum of B_i^2 over the aggregate's rows in increasing order)
// (par_candidates.cpp:124-140, 176-188); Tt is T transposed, whose rows list
// fine rows in increasing order.
__global__ void k_tent_norms(int nc, const int* __restrict__ ttp, const double* __restrict__ ttv,
                             double* R, double* scale) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nc) return;
    double s = 0.0;
    for (int j = ttp[a]; j < ttp[a + 1]; j++) s = dadd(s, dmul(ttv[j], ttv[j]));
    const double ra = __dsqrt_rn(s);
    R[a] = ra;
    scale[a] = __ddiv_rn(1.0, ra);
}

__global__ void k_tent_scale(long long nnz, const int* __restrict__ tci,
                             const double* __restrict__ scale, double* tcv) {
    long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < nnz) tcv[j] = dmul(tcv[j], scale[tci[j]]);
}

// =================================================== jacobi_prolongation ===
// scaled_A = omega D_abs^-1 A, D_abs = sum_j |a_ij| in stored order
// (par_prolongation.cpp:24-54).
__global__ void k_scale_rows_abs(int n, const int* __restrict__ rp, const double* __restrict__ v,
                                 double omega, double* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double row_sum = 0.0;
    for (int j = rp[i]; j < rp[i + 1]; j++) row_sum = dadd(row_sum, fabs(v[j]));
    const double inv = row_sum != 0.0 ? dmul(__ddiv_rn(1.0, fabs(row_sum)), omega) : 0.0;
    for (int j = rp[i]; j < rp[i + 1]; j++) out[j] = dmul(v[j], inv);
}

// P - AP (ParCSRMatrix::subtract): the row of P followed by the negated row
// of AP, stably sorted by column, duplicates summed and |v| < 1e-16 dropped
// (core/matrix.cpp remove_duplicates), then the diagonal moved first.  Each
// column occurs at most once in P's row and once in AP's (sorted, summed)
// row, so a column's value is p, -ap, or p + (-ap) in that order.
template <bool WRITE>
__global__ void k_subtract(int n, const int* __restrict__ prp, const int* __restrict__ pci,
                           const double* __restrict__ pcv, const int* __restrict__ qrp,
                           const int* __restrict__ qci, const double* __restrict__ qcv, int* cnt,
                           const int* __restrict__ crp, int* cci, double* ccv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int ps = prp[i], pe = prp[i + 1], qs = qrp[i], qe = qrp[i + 1];
    int out = WRITE ? crp[i] : 0;
    int m = 0;
    // P's row may be in any order (diagonal first); AP's is sorted.  For
    // each output column in increasing order: find it in both rows.
    int last = INT_MIN;
    while (true) {
        // next column above `last` among both rows
        int c = INT_MAX;
        for (int j = ps; j < pe; j++) { const int x = pci[j]; if (x > last && x < c) c = x; }
        for (int j = qs; j < qe; j++) { const int x = qci[j]; if (x > last) { if (x < c) c = x; break; } }
        if (c == INT_MAX) break;
        bool have = false;
        double v = 0.0;
        for (int j = ps; j < pe; j++)
            if (pci[j] == c) { v = pcv[j]; have = true; break; }
        for (int j = qs; j < qe; j++) {
            if (qci[j] == c) { v = have ? dadd(v, -qcv[j]) : -qcv[j]; break; }
            if (qci[j] > c) break;
        }
        if (fabs(v) >= kZeroTol) {
            if (WRITE) { cci[out + m] = c; ccv[out + m] = v; }
            m++;
        }
        last = c;
    }
    if (!WRITE) cnt[i] = m;
}

}  // namespace

// --------------------------------------------------------------- host ----

void mis2(const rb_csr_s& S, const double* r_dev, int* states_dev) {
    const int n = S.n_rows;
    if (n == 0) return;
    const unsigned g = grid_for(n, 256);
    DevArray<int> st2((size_t)n), C((size_t)n), listed((size_t)n), fresh((size_t)n), rem(1);
    DevArray<double> row_max((size_t)n);
    k_fill_int<<<g, 256, 0, stream()>>>(n, states_dev, kUnassigned);
    RB_CHECK_LAUNCH();
    C.zero();
    listed.zero();
    const int* rp = S.rowptr.get();
    const int* ci = S.cols.get();
    // the reference's loop ends when no node remains; a pass always settles
    // at least the remaining node of largest weight, so n + 1 passes bound it
    for (int pass = 0; pass <= n; pass++) {
        k_mis2_tmp<<<g, 256, 0, stream()>>>(n, rp, ci, r_dev, states_dev, st2.get());
        RB_CHECK_LAUNCH();
        k_mis2_rowmax<<<g, 256, 0, stream()>>>(n, rp, ci, r_dev, st2.get(), row_max.get());
        RB_CHECK_LAUNCH();
        k_mis2_select<<<g, 256, 0, stream()>>>(n, rp, ci, r_dev, row_max.get(), st2.get());
        RB_CHECK_LAUNCH();
        k_mis2_mark<<<g, 256, 0, stream()>>>(n, rp, ci, st2.get(), C.get(), listed.get(),
                                             fresh.get());
        RB_CHECK_LAUNCH();
        k_mis2_unselect<<<g, 256, 0, stream()>>>(n, rp, ci, st2.get(), C.get(), states_dev);
        RB_CHECK_LAUNCH();
        rem.zero();
        k_mis2_commit<<<g, 256, 0, stream()>>>(n, states_dev, C.get(), listed.get(), fresh.get(),
                                               rem.get());
        RB_CHECK_LAUNCH();
        if (read_scalar(rem.get()) == 0) return;
    }
    throw Error(RB_ERR_INVALID, "mis2 did not terminate");
}

int aggregate(const rb_csr_s& A, const rb_csr_s& S, const int* states_dev, int* agg_dev,
              const double* r_dev) {
    const int n = S.n_rows;
    RB_REQUIRE(A.n_rows == n, "aggregate: A and S differ in size");
    if (n == 0) return 0;
    const unsigned g = grid_for(n, 256);
    DevArray<int> counters(3), snap((size_t)n);
    counters.zero();
    k_agg_init<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), states_dev, agg_dev, counters.get());
    RB_CHECK_LAUNCH();
    k_agg_pass1<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), S.cols.get(), states_dev, agg_dev);
    RB_CHECK_LAUNCH();
    RB_CUDA(cudaMemcpyAsync(snap.get(), agg_dev, sizeof(int) * n, cudaMemcpyDeviceToDevice,
                            stream()));
    k_agg_pass2<<<g, 256, 0, stream()>>>(n, A.rowptr.get(), A.cols.get(), A.vals.get(),
                                         S.rowptr.get(), S.cols.get(), r_dev, snap.get(), agg_dev,
                                         counters.get() + 1, counters.get() + 2);
    RB_CHECK_LAUNCH();
    int h[3];
    counters.download(h, 3);
    RB_CUDA(cudaStreamSynchronize(stream()));
    RB_REQUIRE(h[2] == 0, "aggregate: a strong connection is missing from A's row");
    if (h[1] > 0) {
        // rows without any assigned neighbour: their code is visible to later
        // rows in the sequential loop, so run that loop as written
        RB_CUDA(cudaMemcpyAsync(agg_dev, snap.get(), sizeof(int) * n, cudaMemcpyDeviceToDevice,
                                stream()));
        k_agg_pass2_seq<<<1, 1, 0, stream()>>>(n, A.rowptr.get(), A.cols.get(), A.vals.get(),
                                               S.rowptr.get(), S.cols.get(), r_dev, agg_dev,
                                               counters.get() + 2);
        RB_CHECK_LAUNCH();
    }
    k_agg_final<<<g, 256, 0, stream()>>>(n, agg_dev);
    RB_CHECK_LAUNCH();
    return h[0];
}

rb_csr_s* fit_candidates(int n, int n_aggs, const int* agg_dev, const double* B_dev,
                         double* R_dev) {
    const unsigned g = grid_for(n, 256);
    DevArray<int> used((size_t)n + 1), has((size_t)n + 1), cidx((size_t)n + 1);
    used.zero();
    if (n)
        k_mark_used<<<g, 256, 0, stream()>>>(n, agg_dev, used.get(), has.get());
    RB_CHECK_LAUNCH();
    const long long nc = exclusive_scan(used.get(), cidx.get(), n);
    RB_REQUIRE(nc == n_aggs, "fit_candidates: aggregates do not match the number of roots");
    rb_csr_s* T = new_csr(n, n_aggs, 0);
    const long long nnz = exclusive_scan(has.get(), T->rowptr.get(), n);
    T->nnz = nnz;
    T->cols.alloc((size_t)std::max<long long>(nnz, 1));
    T->vals.alloc((size_t)std::max<long long>(nnz, 1));
    if (n)
        k_tent_fill<<<g, 256, 0, stream()>>>(n, agg_dev, cidx.get(), T->rowptr.get(), B_dev,
                                             T->cols.get(), T->vals.get());
    RB_CHECK_LAUNCH();
    if (n_aggs) {
        std::unique_ptr<rb_csr_s> Tt(transpose(*T));
        DevArray<double> scale((size_t)n_aggs);
        k_tent_norms<<<grid_for(n_aggs, 256), 256, 0, stream()>>>(
            n_aggs, Tt->rowptr.get(), Tt->vals.get(), R_dev, scale.get());
        RB_CHECK_LAUNCH();
        if (nnz)
            k_tent_scale<<<grid_for(nnz, 256), 256, 0, stream()>>>(nnz, T->cols.get(),
                                                                  scale.get(), T->vals.get());
        RB_CHECK_LAUNCH();
        RB_CUDA(cudaStreamSynchronize(stream()));
    }
    return T;
}

rb_csr_s* jacobi_prolongation(const rb_csr_s& A, const rb_csr_s& T, double omega, int steps) {
    const int n = A.n_rows;
    RB_REQUIRE(T.n_rows == n && A.n_cols == n, "jacobi_prolongation: sizes differ");
    std::unique_ptr<rb_csr_s> sA(new_csr(n, A.n_cols, A.nnz));
    RB_CUDA(cudaMemcpyAsync(sA->rowptr.get(), A.rowptr.get(), sizeof(int) * (n + 1),
                            cudaMemcpyDeviceToDevice, stream()));
    if (A.nnz)
        RB_CUDA(cudaMemcpyAsync(sA->cols.get(), A.cols.get(), sizeof(int) * A.nnz,
                                cudaMemcpyDeviceToDevice, stream()));
    if (n)
        k_scale_rows_abs<<<grid_for(n, 256), 256, 0, stream()>>>(n, A.rowptr.get(), A.vals.get(),
                                                                omega, sA->vals.get());
    RB_CHECK_LAUNCH();
    // P = T (copy)
    std::unique_ptr<rb_csr_s> P(new_csr(T.n_rows, T.n_cols, T.nnz));
    RB_CUDA(cudaMemcpyAsync(P->rowptr.get(), T.rowptr.get(), sizeof(int) * (n + 1),
                            cudaMemcpyDeviceToDevice, stream()));
    if (T.nnz) {
        RB_CUDA(cudaMemcpyAsync(P->cols.get(), T.cols.get(), sizeof(int) * T.nnz,
                                cudaMemcpyDeviceToDevice, stream()));
        RB_CUDA(cudaMemcpyAsync(P->vals.get(), T.vals.get(), sizeof(double) * T.nnz,
                                cudaMemcpyDeviceToDevice, stream()));
    }
    for (int s = 0; s < steps; s++) {
        std::unique_ptr<rb_csr_s> AP(spgemm(*sA, *P));   // sorted, |v| <= 1e-16 dropped
        DevArray<int> cnt((size_t)n + 1);
        const unsigned g = grid_for(n, 256);
        if (n)
            k_subtract<false><<<g, 256, 0, stream()>>>(
                n, P->rowptr.get(), P->cols.get(), P->vals.get(), AP->rowptr.get(),
                AP->cols.get(), AP->vals.get(), cnt.get(), nullptr, nullptr, nullptr);
        RB_CHECK_LAUNCH();
        rb_csr_s* C = new_csr(n, T.n_cols, 0);
        const long long nnz = exclusive_scan(cnt.get(), C->rowptr.get(), n);
        C->nnz = nnz;
        C->cols.alloc((size_t)std::max<long long>(nnz, 1));
        C->vals.alloc((size_t)std::max<long long>(nnz, 1));
        if (n)
            k_subtract<true><<<g, 256, 0, stream()>>>(
                n, P->rowptr.get(), P->cols.get(), P->vals.get(), AP->rowptr.get(),
                AP->cols.get(), AP->vals.get(), nullptr, C->rowptr.get(), C->cols.get(),
                C->vals.get());
        RB_CHECK_LAUNCH();
        sort_rows_diag_first(*C, true);   // rows are sorted; moves the diagonal first
        P.reset(C);
    }
    RB_CUDA(cudaStreamSynchronize(stream()));
    return P.release();
}

}  // namespace rb
