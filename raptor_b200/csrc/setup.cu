// setup.cu -- AMG setup kernels (Ruge-Stuben path), FP64, bit-exact.
//
// Compiled with -fmad=false, and every accumulation spells out __dmul_rn /
// __dadd_rn: the reference's -O3 x86-64 build has no FMA, and a one-ulp
// difference in an RAP value can flip a strict strength comparison on the
// next level and change every coarser C/F splitting.  Each kernel keeps the
// reference's per-entry accumulation order.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstdlib>

#include "direct_interp.cuh"
#include "rb_internal.cuh"

namespace rb {

constexpr double kZeroTol = 1e-16;           // core/types.hpp:26
constexpr double kRandMax = 2147483647.0;    // glibc RAND_MAX (par_strength.cpp:78)
constexpr int kSelected = 1, kUnselected = 0, kUnassigned = -1, kNoNeighbors = -2;
constexpr int kNewSelection = 3, kNewUnselection = 2;   // core/types.hpp:31-37

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

std::vector<double> rand_weights(int n, int first_row) {
    // form_rand_weights, multilevel/par_multilevel.hpp:215-225
    std::vector<double> w((size_t)n);
    srand(2448422 + first_row);
    for (int i = 0; i < n; i++) w[i] = double(rand()) / RAND_MAX;
    return w;
}

// ============================================================ strength ===
// classical_strength, par_strength.cpp:8-339.  vars (the unknown-based
// systems form, num_variables > 1; NULL otherwise): only entries between rows
// of one variable take part in the row's scale and can be strong.
__device__ __forceinline__ bool same_var(int i, int j, const int* vars) {
    return vars == nullptr || vars[i] == vars[j];
}

template <bool FILL>
__global__ void k_classical_strength(int n, const int* __restrict__ rp,
                                     const int* __restrict__ ci, const double* __restrict__ cv,
                                     double theta, int* cnt, const int* srp, int* sci,
                                     double* scv, const int* __restrict__ nv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int rs = rp[i], re = rp[i + 1];
    int out = FILL ? srp[i] : 0, k = 0;
    if (re - rs) {
        double diag;
        if (ci[rs] == i) { diag = cv[rs]; rs++; }
        else diag = 0.0;
        double row_scale;
        if (diag < 0.0) {
            row_scale = -kRandMax;
            for (int j = rs; j < re; j++)
                if (same_var(i, ci[j], nv) && cv[j] > row_scale) row_scale = cv[j];
        } else {
            row_scale = kRandMax;
            for (int j = rs; j < re; j++)
                if (same_var(i, ci[j], nv) && cv[j] < row_scale) row_scale = cv[j];
        }
        double thr = dmul(row_scale, theta);
        if (FILL) { sci[out] = i; scv[out] = diag; }
        k = 1;
        for (int j = rs; j < re; j++) {
            double v = cv[j];
            if (same_var(i, ci[j], nv) && (diag < 0 ? (v > thr) : (v < thr))) {
                if (FILL) { sci[out + k] = ci[j]; scv[out + k] = v; }
                k++;
            }
        }
    }
    if (!FILL) cnt[i] = k;
}

// symmetric_strength first pass, par_strength.cpp:385-450
__global__ void k_sym_scales(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ cv, double theta, double* scales,
                             int* neg) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int rs = rp[i], re = rp[i + 1];
    double sc = 0.0;
    int ng = 0;
    if (re - rs) {
        double diag;
        if (ci[rs] == i) { diag = cv[rs]; rs++; }
        else diag = 0.0;
        double row_scale;
        if (diag < 0.0) {
            ng = 1;
            row_scale = -kRandMax;
            for (int j = rs; j < re; j++) if (cv[j] > row_scale) row_scale = cv[j];
        } else {
            row_scale = kRandMax;
            for (int j = rs; j < re; j++) if (cv[j] < row_scale) row_scale = cv[j];
        }
        sc = dmul(row_scale, theta);
    }
    scales[i] = sc;
    neg[i] = ng;
}

// symmetric_strength second pass, par_strength.cpp:457-505: the first entry
// of every non-empty row is kept as the diagonal.
template <bool FILL>
__global__ void k_sym_strength(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                               const double* __restrict__ cv, const double* __restrict__ sc,
                               const int* __restrict__ neg, int* cnt, const int* srp, int* sci,
                               double* scv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int rs = rp[i], re = rp[i + 1];
    int out = FILL ? srp[i] : 0, k = 0;
    if (re - rs) {
        int nd = neg[i];
        double thr = sc[i];
        if (FILL) { sci[out] = i; scv[out] = cv[rs]; }
        rs++;
        k = 1;
        for (int j = rs; j < re; j++) {
            double v = cv[j];
            int c = ci[j];
            if ((nd && v > thr) || (!nd && v < thr) || (neg[c] && v > sc[c]) ||
                (!neg[c] && v < sc[c])) {
                if (FILL) { sci[out + k] = c; scv[out + k] = v; }
                k++;
            }
        }
    }
    if (!FILL) cnt[i] = k;
}

rb_csr_s* strength(const rb_csr_s& A, int kind, double theta, const int* nv) {
    const int n = A.n_rows;
    DevArray<int> cnt((size_t)n + 1);
    const unsigned g = grid_for(n, 256);
    rb_csr_s* S = nullptr;
    if (kind == RB_STRENGTH_CLASSICAL) {
        if (n) k_classical_strength<false><<<g, 256, 0, stream()>>>(
            n, A.rowptr.get(), A.cols.get(), A.vals.get(), theta, cnt.get(), nullptr, nullptr, nullptr,
            nv);
        RB_CHECK_LAUNCH();
        DevArray<int> rp((size_t)n + 1);
        long long nnz = exclusive_scan(cnt.get(), rp.get(), n);
        S = new_csr(n, A.n_cols, nnz);
        S->rowptr = std::move(rp);
        if (n) k_classical_strength<true><<<g, 256, 0, stream()>>>(
            n, A.rowptr.get(), A.cols.get(), A.vals.get(), theta, nullptr, S->rowptr.get(),
            S->cols.get(), S->vals.get(), nv);
        RB_CHECK_LAUNCH();
    } else {
        DevArray<double> sc((size_t)n + 1);
        DevArray<int> neg((size_t)n + 1);
        if (n) k_sym_scales<<<g, 256, 0, stream()>>>(n, A.rowptr.get(), A.cols.get(),
                                                     A.vals.get(), theta, sc.get(), neg.get());
        RB_CHECK_LAUNCH();
        if (n) k_sym_strength<false><<<g, 256, 0, stream()>>>(
            n, A.rowptr.get(), A.cols.get(), A.vals.get(), sc.get(), neg.get(), cnt.get(),
            nullptr, nullptr, nullptr);
        RB_CHECK_LAUNCH();
        DevArray<int> rp((size_t)n + 1);
        long long nnz = exclusive_scan(cnt.get(), rp.get(), n);
        S = new_csr(n, A.n_cols, nnz);
        S->rowptr = std::move(rp);
        if (n) k_sym_strength<true><<<g, 256, 0, stream()>>>(
            n, A.rowptr.get(), A.cols.get(), A.vals.get(), sc.get(), neg.get(), nullptr,
            S->rowptr.get(), S->cols.get(), S->vals.get());
        RB_CHECK_LAUNCH();
    }
    return S;
}

// The variable list of the systems form: row i of the finest level is
// variable i % nv (form_variable_list, par_ruge_stuben_solver.hpp:44-53); the
// next level's list is the C points' variables in order
// (par_ruge_stuben_solver.hpp:124-133).
__global__ void k_vars_init(int n, int nv, int* vars) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) vars[i] = i % nv;
}

__global__ void k_c_flags(int n, const int* __restrict__ st, int* f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f[i] = st[i] == 1 ? 1 : 0;
}

__global__ void k_vars_compact(int n, const int* __restrict__ st, const int* __restrict__ pos,
                               const int* __restrict__ vin, int* vout) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && st[i] == 1) vout[pos[i]] = vin[i];
}

void variables_init(int n, int nv, DevArray<int>& vars) {
    vars.alloc((size_t)std::max(n, 1));
    if (n) k_vars_init<<<grid_for(n, 256), 256, 0, stream()>>>(n, nv, vars.get());
    RB_CHECK_LAUNCH();
}

void variables_coarsen(int n, const int* states_dev, DevArray<int>& vars) {
    DevArray<int> f((size_t)n + 1), pos((size_t)n + 1);
    if (n) k_c_flags<<<grid_for(n, 256), 256, 0, stream()>>>(n, states_dev, f.get());
    RB_CHECK_LAUNCH();
    const long long nc = exclusive_scan(f.get(), pos.get(), n);
    DevArray<int> out((size_t)std::max<long long>(nc, 1));
    if (n) k_vars_compact<<<grid_for(n, 256), 256, 0, stream()>>>(n, states_dev, pos.get(),
                                                                  vars.get(), out.get());
    RB_CHECK_LAUNCH();
    vars = std::move(out);
}

// ================================================================ PMIS ===
// split_pmis / pmis_main_loop, par_cf_splitting.cpp:75-131, 158-309,
// 403-495, 1200-1381.  A round reads only weights (which change only when a
// vertex is assigned, to 0) and writes states, so visiting the unassigned
// vertices in parallel selects the same set as the sequential loop.

// Off-diagonal column lists of S (the leading diagonal is skipped), counts.
__global__ void k_s_colcount(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                             int* cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int s = rp[i], e = rp[i + 1];
    if (s < e && ci[s] == i) s++;
    for (int j = s; j < e; j++) atomicAdd(cnt + ci[j], 1);
}

__global__ void k_s_colfill(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                            int* fill, int* tci) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int s = rp[i], e = rp[i + 1];
    if (s < e && ci[s] == i) s++;
    for (int j = s; j < e; j++) tci[atomicAdd(fill + ci[j], 1)] = i;
}

// set_initial_states (:114-131) + initial_weights (:246-309) + the
// pre-loop filter (:1291-1306).  Each influence adds 1.0 in sequence.
__global__ void k_pmis_init(int n, const int* __restrict__ rp, const int* __restrict__ tp,
                            const double* __restrict__ rnd, double* w, int* st) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int state = (rp[i + 1] - rp[i] > 1) ? kUnassigned : kNoNeighbors;
    double wi = rnd[i];
    for (int k = tp[i]; k < tp[i + 1]; k++) wi = dadd(wi, 1.0);
    if (state == kUnassigned && wi < 1) { state = kUnselected; wi = 0.0; }
    else if (state != kUnassigned) wi = 0.0;
    w[i] = wi;
    st[i] = state;
}

__global__ void k_pmis_select(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                              const int* __restrict__ tp, const int* __restrict__ tci,
                              const double* __restrict__ w, int* st) {
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n || st[u] != kUnassigned) return;
    double wu = w[u];
    int s = rp[u], e = rp[u + 1];
    if (s < e && ci[s] == u) s++;
    for (int j = s; j < e; j++) if (w[ci[j]] > wu) return;
    for (int j = tp[u]; j < tp[u + 1]; j++) if (w[tci[j]] > wu) return;
    st[u] = kNewSelection;
}

__global__ void k_pmis_mark(int n, const int* __restrict__ tp, const int* __restrict__ tci,
                            int* st) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || st[c] != kNewSelection) return;
    for (int j = tp[c]; j < tp[c + 1]; j++) {
        int r = tci[j];
        if (st[r] == kUnassigned) st[r] = kNewUnselection;
    }
}

__global__ void k_pmis_update(int n, double* w, int* st, int* remaining) {
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    int keep = 0;
    if (u < n) {
        int s = st[u];
        if (s == kNewSelection) { w[u] = 0.0; st[u] = kSelected; }
        else if (s == kUnassigned || s == kNewUnselection) {
            if (w[u] < 1.0 || s == kNewUnselection) { w[u] = 0.0; st[u] = kUnselected; }
            else keep = 1;
        }
    }
    keep = __syncthreads_count(keep);
    if (threadIdx.x == 0 && keep) atomicAdd(remaining, keep);
}

// pmis_main_loop's start when the states are already set (HMIS after the
// Ruge-Stuben first pass, par_cf_splitting.cpp:1272-1306): the unassigned
// rows that depend on a selected row become unselected, then the weight
// filter; each influence adds 1.0 in sequence, as in k_pmis_init.
__global__ void k_pmis_keep_mark(int n, const int* __restrict__ tp, const int* __restrict__ tci,
                                 int* st) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || st[c] != kSelected) return;
    for (int j = tp[c]; j < tp[c + 1]; j++)
        if (st[tci[j]] == kUnassigned) st[tci[j]] = kUnselected;
}

__global__ void k_pmis_keep_init(int n, const int* __restrict__ tp, const double* __restrict__ rnd,
                                 double* w, int* st) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double wi = rnd[i];
    for (int k = tp[i]; k < tp[i + 1]; k++) wi = dadd(wi, 1.0);
    if (st[i] == kUnassigned && wi < 1) { st[i] = kUnselected; wi = 0.0; }
    else if (st[i] != kUnassigned) wi = 0.0;
    w[i] = wi;
}

__global__ void k_fill_ones(long long n, int* p) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = 1;
}

__global__ void k_count_state(int n, const int* __restrict__ st, int want, int* count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int hit = i < n && st[i] == want;
    hit = __syncthreads_count(hit);
    if (threadIdx.x == 0 && hit) atomicAdd(count, hit);
}

// Off-diagonal column lists of S (tp, tci).
static void s_transpose(const rb_csr_s& S, DevArray<int>& tp, DevArray<int>& tci) {
    const int n = S.n_rows;
    const unsigned g = grid_for(n, 256);
    DevArray<int> cnt((size_t)n + 1);
    tp.alloc((size_t)n + 1);
    cnt.zero();
    k_s_colcount<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), S.cols.get(), cnt.get());
    RB_CHECK_LAUNCH();
    long long tn = exclusive_scan(cnt.get(), tp.get(), n);
    tci.alloc((size_t)std::max(tn, 1LL));
    RB_CUDA(cudaMemcpyAsync(cnt.get(), tp.get(), sizeof(int) * n, cudaMemcpyDeviceToDevice, stream()));
    k_s_colfill<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), S.cols.get(), cnt.get(), tci.get());
    RB_CHECK_LAUNCH();
}

void split_pmis(const rb_csr_s& S, const double* weights_dev, int* states_dev, bool keep_states) {
    const int n = S.n_rows;
    if (n == 0) return;
    const unsigned g = grid_for(n, 256);
    DevArray<int> tp, tci;
    s_transpose(S, tp, tci);
    DevArray<double> w((size_t)n);
    if (keep_states) {
        k_pmis_keep_mark<<<g, 256, 0, stream()>>>(n, tp.get(), tci.get(), states_dev);
        RB_CHECK_LAUNCH();
        k_pmis_keep_init<<<g, 256, 0, stream()>>>(n, tp.get(), weights_dev, w.get(), states_dev);
    } else {
        k_pmis_init<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), tp.get(), weights_dev, w.get(),
                                             states_dev);
    }
    RB_CHECK_LAUNCH();
    DevArray<int> rem(1);
    for (int round = 0; round < 100000; round++) {
        rem.zero();
        k_pmis_select<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), S.cols.get(), tp.get(), tci.get(),
                                               w.get(), states_dev);
        k_pmis_mark<<<g, 256, 0, stream()>>>(n, tp.get(), tci.get(), states_dev);
        k_pmis_update<<<g, 256, 0, stream()>>>(n, w.get(), states_dev, rem.get());
        RB_CHECK_LAUNCH();
        if (read_scalar(rem.get()) == 0) return;
    }
    throw Error(RB_ERR_INVALID, "PMIS did not terminate");
}

// ================================================================ CLJP ===
// split_cljp / cljp_main_loop at one rank (par_cf_splitting.cpp:32-48,
// 246-309, 403-660, 1200-1227, 1383-1607).  A round selects the unassigned
// rows whose weight no strong neighbour (either direction) exceeds (the
// PMIS selection, k_pmis_select), then removes edges: for every new C point
// c, the edge from each unassigned row of c's row (c depends on it), and the
// edge i -> k between two rows that both depend on c (k unassigned, i not an
// old C point), each removal taking 1.0 off the weight of the row at its
// head; rows whose weight falls below 1 become F points.  Each edge is
// removed at most once (its mark is claimed atomically), and every removal
// subtracts the same 1.0, so the weights, and hence the rounds, do not
// depend on the order the C points are visited in: they are those of the
// reference's sequential loops.

// set_initial_states (:114-131) + initial_weights (:246-309); keep: the
// states are already set (Falgout after Ruge-Stuben), only their weights
// are zeroed.
__global__ void k_cljp_init(int n, const int* __restrict__ rp, const int* __restrict__ tp,
                            const double* __restrict__ rnd, double* w, int* st, int keep) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int state = keep ? st[i] : ((rp[i + 1] - rp[i] > 1) ? kUnassigned : kNoNeighbors);
    double wi = rnd[i];
    for (int k = tp[i]; k < tp[i + 1]; k++) wi = dadd(wi, 1.0);
    w[i] = state == kUnassigned ? wi : 0.0;
    st[i] = state;
}

// update_row_weights (:497-542): the edges of the C points' own rows
__global__ void k_cljp_row_edges(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                 const int* __restrict__ st, int want, int* edge, double* w) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || st[c] != want) return;
    int s = rp[c], e = rp[c + 1];
    if (s < e && ci[s] == c) s++;
    for (int j = s; j < e; j++) {
        const int idx = ci[j];
        if (st[idx] == kUnassigned && edge[j]) {
            edge[j] = 0;
            atomicAdd(w + idx, -1.0);
        }
    }
}

// update_local_dist2_weights (:544-660): for a C point c, the edges i -> k
// with both i and k depending on c (k unassigned, i not an old C point)
__global__ void k_cljp_dist2_edges(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                   const int* __restrict__ tp, const int* __restrict__ tci,
                                   const int* __restrict__ st, int want, int* edge, double* w) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || st[c] != want) return;
    for (int jj = tp[c]; jj < tp[c + 1]; jj++) {
        const int idx = tci[jj];
        if (st[idx] == kSelected) continue;
        int s = rp[idx], e = rp[idx + 1];
        if (s < e && ci[s] == idx) s++;
        for (int k = s; k < e; k++) {
            const int idk = ci[k];
            if (st[idk] != kUnassigned || !edge[k]) continue;
            // does idk depend on c (c in idk's row, diagonal excluded)?
            int s2 = rp[idk], e2 = rp[idk + 1];
            if (s2 < e2 && ci[s2] == idk) s2++;
            bool dep = false;
            for (int q = s2; q < e2 && !dep; q++) dep = ci[q] == c;
            if (dep && atomicExch(edge + k, 0) == 1) atomicAdd(w + idk, -1.0);
        }
    }
}

void split_cljp(const rb_csr_s& S, const double* weights_dev, int* states_dev, bool keep_states) {
    const int n = S.n_rows;
    if (n == 0) return;
    const unsigned g = grid_for(n, 256);
    DevArray<int> tp, tci;
    s_transpose(S, tp, tci);
    DevArray<int> edge((size_t)std::max<long long>(S.nnz, 1));
    k_fill_ones<<<grid_for(std::max<long long>(S.nnz, 1), 256), 256, 0, stream()>>>(
        std::max<long long>(S.nnz, 1), edge.get());
    RB_CHECK_LAUNCH();
    DevArray<double> w((size_t)n);
    k_cljp_init<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), tp.get(), weights_dev, w.get(),
                                         states_dev, keep_states ? 1 : 0);
    RB_CHECK_LAUNCH();
    auto remove_edges = [&](int want) {
        k_cljp_row_edges<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), S.cols.get(), states_dev,
                                                  want, edge.get(), w.get());
        RB_CHECK_LAUNCH();
        k_cljp_dist2_edges<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), S.cols.get(), tp.get(),
                                                    tci.get(), states_dev, want, edge.get(),
                                                    w.get());
        RB_CHECK_LAUNCH();
    };
    // C points already set (Falgout) remove their edges before the loop
    if (keep_states) remove_edges(kSelected);
    DevArray<int> rem(1);
    for (int round = 0; round < 100000; round++) {
        rem.zero();
        k_count_state<<<g, 256, 0, stream()>>>(n, states_dev, kUnassigned, rem.get());
        RB_CHECK_LAUNCH();
        if (read_scalar(rem.get()) == 0) return;
        rem.zero();
        k_pmis_select<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), S.cols.get(), tp.get(), tci.get(),
                                               w.get(), states_dev);
        RB_CHECK_LAUNCH();
        remove_edges(kNewSelection);
        k_pmis_update<<<g, 256, 0, stream()>>>(n, w.get(), states_dev, rem.get());
        RB_CHECK_LAUNCH();
    }
    throw Error(RB_ERR_INVALID, "CLJP did not terminate");
}

// ======================================================= interpolation ===
__global__ void k_flag_selected(int n, const int* __restrict__ st, int* f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f[i] = st[i] == kSelected ? 1 : 0;
}

// Position of column c within [lo, hi) of an unsorted list, or -1.
__device__ __forceinline__ int find_in(const int* list, int lo, int hi, int c) {
    for (int t = lo; t < hi; t++)
        if (list[t] == c) return t;
    return -1;
}

// --- mod_classical_interpolation, par_interpolation.cpp:991-1451 --------
__global__ void k_modclass_count(int n, const int* __restrict__ srp, const int* __restrict__ sci,
                                 const int* __restrict__ st, int* cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (st[i] == kSelected) { cnt[i] = 1; return; }
    int k = 0;
    for (int j = srp[i] + 1; j < srp[i + 1]; j++) k += st[sci[j]] == kSelected;
    cnt[i] = k;
}

// direct interpolation (direct_interp.cuh), one thread per row
__global__ void k_direct_count(int n, const int* __restrict__ srp, const int* __restrict__ sci,
                               const int* __restrict__ st, int* cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) cnt[i] = direct_row_count(i, srp, sci, st);
}

__global__ void k_direct_fill(int n, const int* __restrict__ arp, const int* __restrict__ aci,
                              const double* __restrict__ acv, const int* __restrict__ srp,
                              const int* __restrict__ sci, const int* __restrict__ st,
                              const int* __restrict__ prp, int* pcols, double* pvals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) direct_row_fill(i, arp, aci, acv, srp, sci, st, prp[i], pcols, pvals);
}

// pcols holds fine column indices while the row is assembled.
__global__ void k_modclass_fill(int n, const int* __restrict__ arp, const int* __restrict__ aci,
                                const double* __restrict__ acv, const int* __restrict__ srp,
                                const int* __restrict__ sci, const double* __restrict__ scv,
                                const int* __restrict__ st, const int* __restrict__ prp,
                                int* pcols, double* pvals, const int* __restrict__ nv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p0 = prp[i];
    if (st[i] == kSelected) { pcols[p0] = i; pvals[p0] = 1.0; return; }
    int m = p0;
    for (int j = srp[i] + 1; j < srp[i + 1]; j++) {
        int c = sci[j];
        if (st[c] == kSelected) { pcols[m] = c; pvals[m] = scv[j]; m++; }
    }
    const int p1 = m;
    int start = arp[i], end = arp[i + 1];
    if (start >= end) return;
    int ctr = srp[i] + 1, end_S = srp[i + 1];
    double weak_sum = acv[start++];
    for (int j = start; j < end; j++) {
        int col = aci[j];
        double val = acv[j];
        if (ctr < end_S && sci[ctr] == col) {
            ctr++;
            if (st[col] == kSelected) continue;
            double coarse_sum = 0;
            int sk = arp[col], ek = arp[col + 1];
            double diag = acv[sk++];
            int sign = diag > 0 ? 1 : -1;
            for (int k = sk; k < ek; k++) {
                int ck = aci[k];
                if (st[ck] == kSelected) {
                    double vk = acv[k];
                    if (dmul(vk, (double)sign) < 0 && find_in(pcols, p0, p1, ck) >= 0)
                        coarse_sum = dadd(coarse_sum, vk);
                }
            }
            if (fabs(coarse_sum) < kZeroTol) weak_sum = dadd(weak_sum, val);
            else coarse_sum = __ddiv_rn(val, coarse_sum);
            if (coarse_sum != 0.0) {
                for (int k = arp[col] + 1; k < ek; k++) {
                    int ck = aci[k];
                    if (st[ck] == kSelected) {
                        double vk = acv[k];
                        if (dmul(vk, (double)sign) < 0) {
                            int idx = find_in(pcols, p0, p1, ck);
                            if (idx >= 0) pvals[idx] = dadd(pvals[idx], dmul(coarse_sum, vk));
                        }
                    }
                }
            }
        } else if (st[col] != kNoNeighbors && same_var(i, col, nv)) {
            weak_sum = dadd(weak_sum, val);
        }
    }
    for (int t = p0; t < p1; t++) pvals[t] = __ddiv_rn(pvals[t], -weak_sum);
}

// --- extended_interpolation, par_interpolation.cpp:280-989 ---------------
// rows whose C set fits kExtSlots registers a lane go through the warp
// kernels below; larger ones through the one-thread-per-row kernels
constexpr int kExtSlots = 8;
constexpr int kExtWarpMax = 32 * kExtSlots;

// Upper bound of a row's pattern: strong C neighbours plus the strong C
// neighbours of every strong F neighbour.
__global__ void k_ext_bound(int n, const int* __restrict__ srp, const int* __restrict__ sci,
                            const int* __restrict__ st, int* ub) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (st[i] != kUnselected) { ub[i] = 1; return; }
    int b = 0;
    for (int j = srp[i] + 1; j < srp[i + 1]; j++) {
        int c = sci[j];
        if (st[c] == kSelected) b++;
        else if (st[c] == kUnselected) b += srp[c + 1] - srp[c] - 1;
    }
    ub[i] = b;
}

// Insertion-ordered unique pattern (par_interpolation.cpp:574-690) of
// the rows [r0, r0 + n), built in a scratch list to count it.
__device__ __forceinline__ int ext_build_pattern(int i, const int* __restrict__ srp,
                                                 const int* __restrict__ sci,
                                                 const int* __restrict__ st, int* list, int o) {
    int m = o;
    for (int j = srp[i] + 1; j < srp[i + 1]; j++) {
        int c = sci[j];
        if (st[c] == kSelected) {
            if (find_in(list, o, m, c) < 0) list[m++] = c;
        } else if (st[c] == kUnselected) {
            for (int k = srp[c] + 1; k < srp[c + 1]; k++) {
                int ck = sci[k];
                if (st[ck] == kSelected && find_in(list, o, m, ck) < 0) list[m++] = ck;
            }
        }
    }
    return m - o;
}

__global__ void k_ext_pattern(int n, int r0, const int* __restrict__ srp,
                              const int* __restrict__ sci, const int* __restrict__ st,
                              const int* __restrict__ big, const int* __restrict__ uoff, int* list,
                              int* cnt) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = r0 + t;
    const int o = uoff[t];
    if (!big[i]) return;   // counted by k_ext_pattern_warp
    if (st[i] != kUnselected) {
        cnt[i] = st[i] == kSelected ? 1 : 0;
        return;
    }
    cnt[i] = ext_build_pattern(i, srp, sci, st, list, o);
}

// Values (par_interpolation.cpp:692-944) and filter_interp (:175-278).
// The row is assembled in pcols/pvals[prp[i] ...]; kept entries are
// compacted to the front and their count written to kept[i].
__global__ void k_ext_fill(int n, const int* __restrict__ arp, const int* __restrict__ aci,
                           const double* __restrict__ acv, const int* __restrict__ srp,
                           const int* __restrict__ sci, const int* __restrict__ st,
                           const int* __restrict__ prp, int* pcols, double* pvals, double filter,
                           int* kept, const int* __restrict__ nv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p0 = prp[i], p1 = prp[i + 1];
    if (p1 - p0 <= kExtWarpMax) return;   // filled by k_ext_fill_warp
    // rebuild the insertion-ordered pattern in place (its size is p1 - p0)
    if (st[i] == kSelected) pcols[p0] = i;
    else if (st[i] == kUnselected) ext_build_pattern(i, srp, sci, st, pcols, p0);
    for (int t = p0; t < p1; t++) pvals[t] = 0.0;
    if (st[i] == kSelected) { pvals[p0] = 1.0; }
    if (st[i] == kUnselected) {
        int start = arp[i], end = arp[i + 1];
        double weak_sum = acv[start++];
        int ctr = srp[i] + 1, end_S = srp[i + 1];
        for (int j = start; j < end; j++) {
            int col = aci[j];
            double val = acv[j];
            int idx = find_in(pcols, p0, p1, col);
            if (idx >= 0) {
                pvals[idx] = dadd(pvals[idx], val);
                if (ctr < end_S && sci[ctr] == col) ctr++;
            } else if (ctr < end_S && sci[ctr] == col) {
                ctr++;
                if (st[col] != kUnselected) continue;
                double col_sum = 0;
                int sk = arp[col], ek = arp[col + 1];
                double diag = acv[sk++];
                int sign = diag > 0 ? 1 : -1;
                for (int k = sk; k < ek; k++) {
                    double vk = acv[k];
                    int ck = aci[k];
                    if (dmul(vk, (double)sign) < 0 && (ck == i || find_in(pcols, p0, p1, ck) >= 0))
                        col_sum = dadd(col_sum, vk);
                }
                if (fabs(col_sum) < kZeroTol) {
                    weak_sum = dadd(weak_sum, val);
                } else {
                    col_sum = __ddiv_rn(val, col_sum);
                    for (int k = arp[col] + 1; k < ek; k++) {
                        int ck = aci[k];
                        double vk = acv[k];
                        if (dmul(vk, (double)sign) < 0) {
                            if (ck == i) weak_sum = dadd(weak_sum, dmul(col_sum, vk));
                            else {
                                int id = find_in(pcols, p0, p1, ck);
                                if (id >= 0) pvals[id] = dadd(pvals[id], dmul(col_sum, vk));
                            }
                        }
                    }
                }
            } else {
                if (st[col] != kNoNeighbors && same_var(i, col, nv)) weak_sum = dadd(weak_sum, val);
            }
        }
        if (fabs(weak_sum) > kZeroTol)
            for (int t = p0; t < p1; t++) pvals[t] = __ddiv_rn(pvals[t], -weak_sum);
    }
    // filter_interp (only when 0 < filter <= 1)
    int out = p0;
    if (filter > kZeroTol && filter <= 1) {
        double row_max = 0;
        for (int t = p0; t < p1; t++) {
            double a = fabs(pvals[t]);
            if (a > row_max) row_max = a;
        }
        row_max = dmul(row_max, filter);
        double row_sum = 0, remain_sum = 0;
        for (int t = p0; t < p1; t++) {
            double v = pvals[t];
            row_sum = dadd(row_sum, v);
            if (fabs(v) >= row_max) {
                pcols[out] = pcols[t];
                pvals[out] = v;
                out++;
                remain_sum = dadd(remain_sum, v);
            }
        }
        if (fabs(remain_sum) > kZeroTol && fabs(dsub(row_sum, remain_sum)) > kZeroTol) {
            double scale = __ddiv_rn(row_sum, remain_sum);
            for (int t = p0; t < out; t++) pvals[t] = dmul(pvals[t], scale);
        }
    } else {
        out = p1;
    }
    kept[i] = out - p0;
}

// ---- warp-per-row extended interpolation -------------------------------
// The same arithmetic, in the same order, as k_ext_pattern / k_ext_fill,
// with one warp per row.  The row's insertion-ordered C set, a hash table
// from column to position and the weights live in the warp's shared memory.
// Loops over a neighbour's row run one entry per lane: membership tests are
// parallel hash probes, new C points are appended in entry order (ballot
// prefix), the weights of one neighbour's expansion go to distinct
// positions, and every sum whose order matters (col_sum, weak_sum, the
// filter's row sums) is folded sequentially in the original order.  Rows
// whose set exceeds kExtWarpMax entries take the one-thread-per-row kernels.
constexpr int kExtHash = 2 * kExtWarpMax;   // hash slots per warp
constexpr int kExtWarps = 8;                // warps per block

struct ExtWarpMem {
    int keys[kExtHash];
    int pos[kExtHash];
    int list[kExtWarpMax];
    double vals[kExtWarpMax];
};

__device__ __forceinline__ unsigned ext_hash(int c) { return (unsigned)c * 2654435761u; }

// position of column c in the set, or -1
__device__ __forceinline__ int ext_find(const ExtWarpMem& w, int c) {
    unsigned h = ext_hash(c) & (kExtHash - 1);
    while (true) {
        const int k = w.keys[h];
        if (k == c) return w.pos[h];
        if (k == -1) return -1;
        h = (h + 1) & (kExtHash - 1);
    }
}

// insert column c (not yet present) at position p; distinct keys may be
// inserted by several lanes at once
__device__ __forceinline__ void ext_insert(ExtWarpMem& w, int c, int p) {
    unsigned h = ext_hash(c) & (kExtHash - 1);
    while (true) {
        if (atomicCAS(&w.keys[h], -1, c) == -1) {
            w.pos[h] = p;
            return;
        }
        h = (h + 1) & (kExtHash - 1);
    }
}

// Insertion-ordered C set of row i; returns its size, or kExtWarpMax + 1
// when it does not fit.
__device__ int ext_build_warp(int i, const int* __restrict__ srp, const int* __restrict__ sci,
                              const int* __restrict__ st, ExtWarpMem& w, int lane) {
    for (int t = lane; t < kExtHash; t += 32) w.keys[t] = -1;
    __syncwarp();
    int m = 0;
    for (int j = srp[i] + 1; j < srp[i + 1]; j++) {
        const int c = sci[j];
        const int sc = st[c];
        if (sc == kSelected) {
            if (ext_find(w, c) < 0) {
                if (m >= kExtWarpMax) return kExtWarpMax + 1;
                if (lane == 0) {
                    w.list[m] = c;
                    ext_insert(w, c, m);
                }
                m++;
                __syncwarp();
            }
        } else if (sc == kUnselected) {
            for (int base = srp[c] + 1; base < srp[c + 1]; base += 32) {
                const int k = base + lane;
                const int ck = k < srp[c + 1] ? sci[k] : -1;
                const bool isnew = ck >= 0 && st[ck] == kSelected && ext_find(w, ck) < 0;
                const unsigned b = __ballot_sync(0xffffffffu, isnew);
                const int add = __popc(b);
                if (m + add > kExtWarpMax) return kExtWarpMax + 1;
                if (isnew) {
                    const int p = m + __popc(b & ((1u << lane) - 1));
                    w.list[p] = ck;
                    ext_insert(w, ck, p);
                }
                m += add;
                __syncwarp();
            }
        }
    }
    return m;
}

// Pattern sizes of the rows whose C set fits; a row that does not is marked
// (big[i] = 1) for the one-thread-per-row kernel.
__global__ void __launch_bounds__(kExtWarps * 32)
k_ext_pattern_warp(int n, const int* __restrict__ srp, const int* __restrict__ sci,
                   const int* __restrict__ st, int* cnt, int* big) {
    extern __shared__ unsigned char ext_smem[];
    ExtWarpMem& w = reinterpret_cast<ExtWarpMem*>(ext_smem)[threadIdx.x >> 5];
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= n) return;
    if (st[i] != kUnselected) {
        if (lane == 0) { cnt[i] = st[i] == kSelected ? 1 : 0; big[i] = 0; }
        return;
    }
    const int m = ext_build_warp(i, srp, sci, st, w, lane);
    if (lane == 0) {
        big[i] = m > kExtWarpMax ? 1 : 0;
        if (m <= kExtWarpMax) cnt[i] = m;
    }
}

__global__ void __launch_bounds__(kExtWarps * 32)
k_ext_fill_warp(int n, const int* __restrict__ arp, const int* __restrict__ aci,
                const double* __restrict__ acv, const int* __restrict__ srp,
                const int* __restrict__ sci, const int* __restrict__ st,
                const int* __restrict__ prp, int* pcols, double* pvals, double filter,
                int* kept, const int* __restrict__ nv) {
    extern __shared__ unsigned char ext_smem[];
    ExtWarpMem& w = reinterpret_cast<ExtWarpMem*>(ext_smem)[threadIdx.x >> 5];
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= n) return;
    const int p0 = prp[i], p1 = prp[i + 1];
    if (p1 - p0 > kExtWarpMax) return;   // the one-thread-per-row kernel takes it
    const int si = st[i];
    int m = 0;
    if (si == kSelected) {
        if (lane == 0) { w.list[0] = i; w.vals[0] = 1.0; }
        m = 1;
        __syncwarp();
    } else if (si == kUnselected) {
        m = ext_build_warp(i, srp, sci, st, w, lane);
        for (int t = lane; t < m; t += 32) w.vals[t] = 0.0;
        __syncwarp();
        int start = arp[i];
        const int end = arp[i + 1];
        double weak_sum = acv[start++];
        int ctr = srp[i] + 1;
        const int end_S = srp[i + 1];
        for (int j = start; j < end; j++) {
            const int col = aci[j];
            const double val = acv[j];
            const int idx = ext_find(w, col);
            if (idx >= 0) {
                if (lane == 0) w.vals[idx] = dadd(w.vals[idx], val);
                __syncwarp();
                if (ctr < end_S && sci[ctr] == col) ctr++;
            } else if (ctr < end_S && sci[ctr] == col) {
                ctr++;
                if (st[col] != kUnselected) continue;
                const int sk = arp[col] + 1, ek = arp[col + 1];
                const int sign = acv[arp[col]] > 0 ? 1 : -1;
                // col_sum: the qualifying entries of row col, summed in order
                double col_sum = 0;
                for (int base = sk; base < ek; base += 32) {
                    const int k = base + lane;
                    double vk = 0.0;
                    bool q = false;
                    if (k < ek) {
                        vk = acv[k];
                        const int ck = aci[k];
                        q = dmul(vk, (double)sign) < 0 && (ck == i || ext_find(w, ck) >= 0);
                    }
                    unsigned b = __ballot_sync(0xffffffffu, q);
                    while (b) {
                        const int t = __ffs(b) - 1;
                        col_sum = dadd(col_sum, __shfl_sync(0xffffffffu, vk, t));
                        b &= b - 1;
                    }
                }
                if (fabs(col_sum) < kZeroTol) {
                    weak_sum = dadd(weak_sum, val);
                } else {
                    col_sum = __ddiv_rn(val, col_sum);
                    for (int base = sk; base < ek; base += 32) {
                        const int k = base + lane;
                        bool self = false;
                        double term = 0.0;
                        if (k < ek) {
                            const int ck = aci[k];
                            const double vk = acv[k];
                            if (dmul(vk, (double)sign) < 0) {
                                term = dmul(col_sum, vk);
                                if (ck == i) {
                                    self = true;
                                } else {
                                    const int id = ext_find(w, ck);
                                    if (id >= 0) w.vals[id] = dadd(w.vals[id], term);
                                }
                            }
                        }
                        // i occurs at most once in row col: its term joins
                        // weak_sum at its place in the sequence
                        const unsigned sb = __ballot_sync(0xffffffffu, self);
                        if (sb) weak_sum = dadd(weak_sum, __shfl_sync(0xffffffffu, term, __ffs(sb) - 1));
                    }
                    __syncwarp();
                }
            } else {
                if (st[col] != kNoNeighbors && same_var(i, col, nv)) weak_sum = dadd(weak_sum, val);
            }
        }
        if (fabs(weak_sum) > kZeroTol)
            for (int t = lane; t < m; t += 32) w.vals[t] = __ddiv_rn(w.vals[t], -weak_sum);
        __syncwarp();
    }
    // filter_interp (only when 0 < filter <= 1), then the kept entries in order
    const bool filt = filter > kZeroTol && filter <= 1;
    double row_max = 0;
    double scale = 1.0;
    bool rescale = false;
    if (filt) {
        for (int t = lane; t < m; t += 32) row_max = fmax(row_max, fabs(w.vals[t]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) row_max = fmax(row_max, __shfl_xor_sync(0xffffffffu, row_max, o));
        row_max = dmul(row_max, filter);
        double row_sum = 0, remain_sum = 0;
        for (int t = 0; t < m; t++) {
            const double v = w.vals[t];
            row_sum = dadd(row_sum, v);
            if (fabs(v) >= row_max) remain_sum = dadd(remain_sum, v);
        }
        if (fabs(remain_sum) > kZeroTol && fabs(dsub(row_sum, remain_sum)) > kZeroTol) {
            scale = __ddiv_rn(row_sum, remain_sum);
            rescale = true;
        }
    }
    int out = 0;
    for (int base = 0; base < m; base += 32) {
        const int t = base + lane;
        const double v = t < m ? w.vals[t] : 0.0;
        const bool keep = t < m && (!filt || fabs(v) >= row_max);
        const unsigned b = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const int pos = p0 + out + __popc(b & ((1u << lane) - 1));
            pcols[pos] = w.list[t];
            pvals[pos] = rescale ? dmul(v, scale) : v;
        }
        out += __popc(b);
    }
    if (lane == 0) kept[i] = out;
}

// Copy the first kept[i] entries of each row, mapping fine C columns to their
// coarse index, and sort the row by column.
__global__ void k_compact_rows(int n, const int* __restrict__ srcp, const int* __restrict__ scol,
                               const double* __restrict__ sval, const int* __restrict__ dstp,
                               const int* __restrict__ cmap, int* dcol, double* dval) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int s = srcp[i], d = dstp[i], m = dstp[i + 1] - d;
    for (int t = 0; t < m; t++) {
        int c = cmap[scol[s + t]];
        double v = sval[s + t];
        int k = t - 1;
        while (k >= 0 && dcol[d + k] > c) {
            dcol[d + k + 1] = dcol[d + k];
            dval[d + k + 1] = dval[d + k];
            k--;
        }
        dcol[d + k + 1] = c;
        dval[d + k + 1] = v;
    }
}

rb_csr_s* interpolation(const rb_csr_s& A, const rb_csr_s& S, const int* st, int kind,
                        double filter, const int* nv) {
    const int n = A.n_rows;
    RB_REQUIRE(S.n_rows == n, "strength matrix does not match A");
    const unsigned g = grid_for(n, 256);
    DevArray<int> flag((size_t)n + 1), cmap((size_t)n + 1);
    if (n) k_flag_selected<<<g, 256, 0, stream()>>>(n, st, flag.get());
    RB_CHECK_LAUNCH();
    const int nc = (int)exclusive_scan(flag.get(), cmap.get(), n);
    DevArray<int> cnt((size_t)n + 1), prp((size_t)n + 1), kept((size_t)n + 1);
    DevArray<int> pcols;
    DevArray<double> pvals;
    if (kind == RB_INTERP_DIRECT) {
        if (n) k_direct_count<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), S.cols.get(), st, cnt.get());
        RB_CHECK_LAUNCH();
        long long nnz = exclusive_scan(cnt.get(), prp.get(), n);
        rb_csr_s* P = new_csr(n, nc, nnz);
        P->rowptr = std::move(prp);
        DevArray<int> fine_cols((size_t)std::max(nnz, 1LL));
        if (n) k_direct_fill<<<g, 256, 0, stream()>>>(
            n, A.rowptr.get(), A.cols.get(), A.vals.get(), S.rowptr.get(), S.cols.get(), st,
            P->rowptr.get(), fine_cols.get(), P->vals.get());
        RB_CHECK_LAUNCH();
        // map to coarse indices (S's rows, and so P's, are in increasing column order)
        DevArray<double> tmpv((size_t)std::max(nnz, 1LL));
        RB_CUDA(cudaMemcpyAsync(tmpv.get(), P->vals.get(), sizeof(double) * nnz,
                                cudaMemcpyDeviceToDevice, stream()));
        if (n) k_compact_rows<<<g, 256, 0, stream()>>>(n, P->rowptr.get(), fine_cols.get(),
                                                       tmpv.get(), P->rowptr.get(), cmap.get(),
                                                       P->cols.get(), P->vals.get());
        RB_CHECK_LAUNCH();
        return P;
    }
    if (kind == RB_INTERP_MODCLASSICAL) {
        if (n) k_modclass_count<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), S.cols.get(), st, cnt.get());
        RB_CHECK_LAUNCH();
        long long nnz = exclusive_scan(cnt.get(), prp.get(), n);
        rb_csr_s* P = new_csr(n, nc, nnz);
        P->rowptr = std::move(prp);
        DevArray<int> fine_cols((size_t)std::max(nnz, 1LL));
        if (n) k_modclass_fill<<<g, 256, 0, stream()>>>(
            n, A.rowptr.get(), A.cols.get(), A.vals.get(), S.rowptr.get(), S.cols.get(),
            S.vals.get(), st, P->rowptr.get(), fine_cols.get(), P->vals.get(), nv);
        RB_CHECK_LAUNCH();
        // map to coarse indices (rows are already in increasing column order)
        DevArray<double> tmpv((size_t)std::max(nnz, 1LL));
        RB_CUDA(cudaMemcpyAsync(tmpv.get(), P->vals.get(), sizeof(double) * nnz,
                                cudaMemcpyDeviceToDevice, stream()));
        if (n) k_compact_rows<<<g, 256, 0, stream()>>>(n, P->rowptr.get(), fine_cols.get(),
                                                       tmpv.get(), P->rowptr.get(), cmap.get(),
                                                       P->cols.get(), P->vals.get());
        RB_CHECK_LAUNCH();
        return P;
    }
    // Extended+i: count each row's pattern in chunks whose dedup scratch
    // (bounded by the row bounds) fits an int32-indexed buffer
    DevArray<int> ub((size_t)n + 1);
    if (n) k_ext_bound<<<g, 256, 0, stream()>>>(n, S.rowptr.get(), S.cols.get(), st, ub.get());
    RB_CHECK_LAUNCH();
    DevArray<int> big((size_t)n + 1);
    RB_CUDA(cudaFuncSetAttribute(k_ext_pattern_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kExtWarps * sizeof(ExtWarpMem))));
    RB_CUDA(cudaFuncSetAttribute(k_ext_fill_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kExtWarps * sizeof(ExtWarpMem))));
    if (n)
        k_ext_pattern_warp<<<grid_for((long)n * 32, kExtWarps * 32), kExtWarps * 32,
                             kExtWarps * sizeof(ExtWarpMem), stream()>>>(
            n, S.rowptr.get(), S.cols.get(), st, cnt.get(), big.get());
    RB_CHECK_LAUNCH();
    std::vector<int> ubh((size_t)n), bigh((size_t)n);
    ub.download(ubh.data(), n);
    big.download(bigh.data(), n);
    RB_CUDA(cudaStreamSynchronize(stream()));
    // scratch only for the rows the warp kernel left
    for (int i = 0; i < n; i++)
        if (!bigh[i]) ubh[i] = 0;
    DevArray<int> ubl((size_t)n + 1);
    ubl.upload(ubh.data(), n);
    const long long kChunk = 1LL << 28;   // 1 GiB of int scratch per chunk
    long long maxchunk = 0;
    {
        long long acc = 0;
        for (int i = 0; i < n; i++) {
            if (acc + ubh[i] > kChunk && acc > 0) { maxchunk = std::max(maxchunk, acc); acc = 0; }
            acc += ubh[i];
        }
        maxchunk = std::max(maxchunk, acc);
    }
    DevArray<int> list((size_t)std::max(maxchunk, 1LL)), uoff((size_t)n + 1);
    for (int r0 = 0; r0 < n;) {
        long long acc = 0;
        int r1 = r0;
        while (r1 < n && (acc + ubh[r1] <= kChunk || r1 == r0)) acc += ubh[r1++];
        const int cn = r1 - r0;
        exclusive_scan(ubl.get() + r0, uoff.get(), cn);
        k_ext_pattern<<<grid_for(cn, 256), 256, 0, stream()>>>(cn, r0, S.rowptr.get(), S.cols.get(),
                                                               st, big.get(), uoff.get(), list.get(),
                                                               cnt.get());
        RB_CHECK_LAUNCH();
        r0 = r1;
    }
    list.release();
    uoff.release();
    ub.release();
    ubl.release();
    long long nnz0 = exclusive_scan(cnt.get(), prp.get(), n);
    pcols.alloc((size_t)std::max(nnz0, 1LL));
    pvals.alloc((size_t)std::max(nnz0, 1LL));
    if (n) {
        k_ext_fill_warp<<<grid_for((long)n * 32, kExtWarps * 32), kExtWarps * 32,
                          kExtWarps * sizeof(ExtWarpMem), stream()>>>(
            n, A.rowptr.get(), A.cols.get(), A.vals.get(), S.rowptr.get(), S.cols.get(), st,
            prp.get(), pcols.get(), pvals.get(), filter, kept.get(), nv);
        RB_CHECK_LAUNCH();
        k_ext_fill<<<g, 256, 0, stream()>>>(
            n, A.rowptr.get(), A.cols.get(), A.vals.get(), S.rowptr.get(), S.cols.get(), st,
            prp.get(), pcols.get(), pvals.get(), filter, kept.get(), nv);
    }
    RB_CHECK_LAUNCH();
    DevArray<int> frp((size_t)n + 1);
    long long nnz = exclusive_scan(kept.get(), frp.get(), n);
    rb_csr_s* P = new_csr(n, nc, nnz);
    P->rowptr = std::move(frp);
    if (n) k_compact_rows<<<g, 256, 0, stream()>>>(n, prp.get(), pcols.get(), pvals.get(),
                                                   P->rowptr.get(), cmap.get(), P->cols.get(),
                                                   P->vals.get());
    RB_CHECK_LAUNCH();
    return P;
}

// ============================================================== SpGEMM ===
// C = A B, one warp per row of A.  spgemm_helper (util/linalg/matmult.cpp
// :71-137) accumulates sums[col] += a_ij * b_jk walking A's row in stored
// order; here the warp walks A's row serially and its lanes split B's row j,
// whose columns are distinct, so every accumulator still receives its terms
// in A's row order and the sums are bit-identical.  |sum| <= 1e-16 is
// dropped; the row is written sorted by column (add_append's sort,
// util/linalg/add.cpp:75).  Pass 1 counts survivors, pass 2 writes them.

__device__ __forceinline__ unsigned hash_col(int c) { return (unsigned)c * 2654435761u; }

// Insert/find column c in an open-addressing table of size H (power of two).
__device__ __forceinline__ int hash_slot(int* keys, int H, int c) {
    unsigned h = hash_col(c) & (H - 1);
    while (true) {
        int k = keys[h];
        if (k == c) return (int)h;
        if (k == -1) {
            int old = atomicCAS(keys + h, -1, c);
            if (old == -1 || old == c) return (int)h;
        }
        h = (h + 1) & (H - 1);
    }
}

template <bool WRITE>
__device__ void spgemm_row(int lane, int row, const int* __restrict__ arp,
                           const int* __restrict__ aci, const double* __restrict__ acv,
                           const int* __restrict__ brp, const int* __restrict__ bci,
                           const double* __restrict__ bcv, int* keys, double* sums, int* clist,
                           int H, int* cnt, const int* crp, int* cci, double* ccv) {
    for (int t = lane; t < H; t += 32) { keys[t] = -1; sums[t] = 0.0; }
    __syncwarp();
    const int as = arp[row], ae = arp[row + 1];
    for (int j = as; j < ae; j++) {
        const int ca = aci[j];
        const double va = acv[j];
        const int bs = brp[ca], be = brp[ca + 1];
        for (int k = bs + lane; k < be; k += 32) {
            const int cb = bci[k];
            const int slot = hash_slot(keys, H, cb);
            sums[slot] = dadd(sums[slot], dmul(va, bcv[k]));
        }
        __syncwarp();
    }
    // compact surviving entries into clist (slot indices), warp-ordered
    int m = 0;
    for (int base = 0; base < H; base += 32) {
        const int t = base + lane;
        const bool keep = keys[t] != -1 && fabs(sums[t]) > kZeroTol;
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (keep) clist[m + __popc(bal & ((1u << lane) - 1))] = t;
        m += __popc(bal);
    }
    __syncwarp();
    if (lane == 0 && cnt) cnt[row] = m;
    if (!WRITE) return;
    // rank by column and write sorted
    const int out = crp[row];
    for (int a = lane; a < m; a += 32) {
        const int sa = clist[a];
        const int c = keys[sa];
        int r = 0;
        for (int b = 0; b < m; b++) r += keys[clist[b]] < c;
        cci[out + r] = c;
        ccv[out + r] = sums[sa];
    }
}

// Structural size of a row of C (distinct columns, before the |v| <= 1e-16
// drop) with key-only hash tables: 4 bytes a slot instead of 16, so four
// times the warps per SM of the numeric pass.
__device__ void spgemm_row_keys(int lane, int row, const int* __restrict__ arp,
                                const int* __restrict__ aci, const int* __restrict__ brp,
                                const int* __restrict__ bci, int* keys, int H, int* scnt) {
    for (int t = lane; t < H; t += 32) keys[t] = -1;
    __syncwarp();
    const int as = arp[row], ae = arp[row + 1];
    for (int j = as; j < ae; j++) {
        const int ca = aci[j];
        const int bs = brp[ca], be = brp[ca + 1];
        for (int k = bs + lane; k < be; k += 32) hash_slot(keys, H, bci[k]);
        __syncwarp();
    }
    int m = 0;
    for (int base = 0; base < H; base += 32)
        m += __popc(__ballot_sync(0xffffffffu, keys[base + lane] != -1));
    if (lane == 0) scnt[row] = m;
}

template <int H, int WPB>
__global__ void __launch_bounds__(WPB * 32)
k_spgemm_keys(const int* __restrict__ rows, int nrows, const int* __restrict__ arp,
              const int* __restrict__ aci, const int* __restrict__ brp,
              const int* __restrict__ bci, int* scnt) {
    extern __shared__ int kmem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int idx = blockIdx.x * WPB + w;
    if (idx >= nrows) return;
    spgemm_row_keys(lane, rows[idx], arp, aci, brp, bci, kmem + (size_t)w * H, H, scnt);
}

__global__ void k_spgemm_keys_global(const int* __restrict__ rows, int nrows,
                                     const long long* __restrict__ toff,
                                     const int* __restrict__ tsize, const int* __restrict__ arp,
                                     const int* __restrict__ aci, const int* __restrict__ brp,
                                     const int* __restrict__ bci, int* gkeys, int* scnt) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nrows) return;
    spgemm_row_keys(lane, rows[w], arp, aci, brp, bci, gkeys + toff[w], tsize[w], scnt);
}

// Bin rows by a size: <= lim0 -> bin 0, <= lim1 -> bin 1, else bin 2.
__global__ void k_bin_rows(int n, const int* __restrict__ size, int lim0, int lim1, int* bins,
                           int* bin_count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int u = size[i];
    const int bin = u <= lim0 ? 0 : (u <= lim1 ? 1 : 2);
    const int p = atomicAdd(bin_count + bin, 1);
    bins[(size_t)bin * n + p] = i;
}

// Move each row's first cnt[i] entries from the capacity layout (cap
// offsets) to the final one (out offsets).
__global__ void k_spgemm_compact(int n, const int* __restrict__ cap, const int* __restrict__ out,
                                 const int* __restrict__ cnt, const int* __restrict__ ci,
                                 const double* __restrict__ cv, int* oci, double* ocv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = cap[i], d = out[i];
    for (int t = 0; t < cnt[i]; t++) {
        oci[d + t] = ci[s + t];
        ocv[d + t] = cv[s + t];
    }
}

template <bool WRITE, int H, int WPB>
__global__ void __launch_bounds__(WPB * 32)
k_spgemm_smem(const int* __restrict__ rows, int nrows, const int* __restrict__ arp,
              const int* __restrict__ aci, const double* __restrict__ acv,
              const int* __restrict__ brp, const int* __restrict__ bci,
              const double* __restrict__ bcv, int* cnt, const int* crp, int* cci, double* ccv) {
    extern __shared__ unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* sums = reinterpret_cast<double*>(smem) + (size_t)w * H;
    int* keys = reinterpret_cast<int*>(reinterpret_cast<double*>(smem) + (size_t)WPB * H) + (size_t)w * 2 * H;
    int* clist = keys + H;
    const int idx = blockIdx.x * WPB + w;
    if (idx >= nrows) return;
    spgemm_row<WRITE>(lane, rows[idx], arp, aci, acv, brp, bci, bcv, keys, sums, clist, H, cnt,
                      crp, cci, ccv);
}

// Rows whose bound exceeds the shared tables: tables in global scratch.
template <bool WRITE>
__global__ void k_spgemm_global(const int* __restrict__ rows, int nrows,
                                const long long* __restrict__ toff, const int* __restrict__ tsize,
                                const int* __restrict__ arp, const int* __restrict__ aci,
                                const double* __restrict__ acv, const int* __restrict__ brp,
                                const int* __restrict__ bci, const double* __restrict__ bcv,
                                int* gkeys, double* gsums, int* glist, int* cnt, const int* crp,
                                int* cci, double* ccv) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nrows) return;
    const long long o = toff[w];
    spgemm_row<WRITE>(lane, rows[w], arp, aci, acv, brp, bci, bcv, gkeys + o, gsums + o, glist + o,
                      tsize[w], cnt, crp, cci, ccv);
}

// Upper bound of the row size of C and the bin of each row.
__global__ void k_spgemm_bound(int n, const int* __restrict__ arp, const int* __restrict__ aci,
                               const int* __restrict__ brp, int* ub, int* bins, int* bin_count,
                               int lim0, int lim1) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long b = 0;
    for (int j = arp[i]; j < arp[i + 1]; j++) b += brp[aci[j] + 1] - brp[aci[j]];
    int u = (int)(b > INT_MAX / 4 ? INT_MAX / 4 : b);
    ub[i] = u;
    int bin = u <= lim0 ? 0 : (u <= lim1 ? 1 : 2);
    int p = atomicAdd(bin_count + bin, 1);
    bins[(size_t)bin * n + p] = i;
}

namespace {
constexpr int kH0 = 512, kW0 = 8;    // 8 warps x (512 x 16 B) = 64 KB
constexpr int kH1 = 4096, kW1 = 2;   // 2 warps x (4096 x 16 B) = 128 KB

inline int next_pow2(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

template <bool WRITE>
void spgemm_pass(const rb_csr_s& A, const rb_csr_s& B, const int* bins, const int* bcount,
                 const std::vector<int>& big_rows_tsize, const DevArray<long long>& toff,
                 const DevArray<int>& tsize, DevArray<int>& gkeys, DevArray<double>& gsums,
                 DevArray<int>& glist, int* cnt, const int* crp, int* cci, double* ccv) {
    const int n = A.n_rows;
    if (bcount[0]) {
        size_t sm = (size_t)kW0 * kH0 * (sizeof(double) + 2 * sizeof(int));
        auto kern = k_spgemm_smem<WRITE, kH0, kW0>;
        RB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        kern<<<grid_for(bcount[0], kW0), kW0 * 32, sm, stream()>>>(
            bins, bcount[0], A.rowptr.get(), A.cols.get(), A.vals.get(), B.rowptr.get(),
            B.cols.get(), B.vals.get(), cnt, crp, cci, ccv);
        RB_CHECK_LAUNCH();
    }
    if (bcount[1]) {
        size_t sm = (size_t)kW1 * kH1 * (sizeof(double) + 2 * sizeof(int));
        auto kern = k_spgemm_smem<WRITE, kH1, kW1>;
        RB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        kern<<<grid_for(bcount[1], kW1), kW1 * 32, sm, stream()>>>(
            bins + (size_t)n, bcount[1], A.rowptr.get(), A.cols.get(), A.vals.get(),
            B.rowptr.get(), B.cols.get(), B.vals.get(), cnt, crp, cci, ccv);
        RB_CHECK_LAUNCH();
    }
    if (bcount[2]) {
        k_spgemm_global<WRITE><<<grid_for((long)bcount[2] * 32, 128), 128, 0, stream()>>>(
            bins + 2 * (size_t)n, bcount[2], toff.get(), tsize.get(), A.rowptr.get(),
            A.cols.get(), A.vals.get(), B.rowptr.get(), B.cols.get(), B.vals.get(), gkeys.get(),
            gsums.get(), glist.get(), cnt, crp, cci, ccv);
        RB_CHECK_LAUNCH();
    }
    (void)big_rows_tsize;
}
}  // namespace

namespace {
constexpr int kK0 = 1024, kKW0 = 16;   // key pass: 16 warps x 1024 x 4 B = 64 KB
constexpr int kK1 = 8192, kKW1 = 4;    // key pass: 4 warps x 8192 x 4 B = 128 KB

// Global tables (one per row of bin 2), sized from a per-row size.
struct GlobalTables {
    DevArray<long long> toff;
    DevArray<int> tsize;
    long long total = 0;
};

GlobalTables global_tables(const int* bins2, int count, const int* size_dev, int n) {
    GlobalTables g;
    if (!count) return g;
    std::vector<int> rows(count), sz_h(n);
    RB_CUDA(cudaMemcpyAsync(rows.data(), bins2, sizeof(int) * count, cudaMemcpyDeviceToHost,
                            stream()));
    RB_CUDA(cudaMemcpyAsync(sz_h.data(), size_dev, sizeof(int) * n, cudaMemcpyDeviceToHost,
                            stream()));
    RB_CUDA(cudaStreamSynchronize(stream()));
    std::vector<long long> off(count);
    std::vector<int> sz(count);
    for (int t = 0; t < count; t++) {
        sz[t] = next_pow2(std::max(64, 2 * sz_h[rows[t]]));
        off[t] = g.total;
        g.total += sz[t];
    }
    g.toff.alloc(count);
    g.toff.upload(off.data(), count);
    g.tsize.alloc(count);
    g.tsize.upload(sz.data(), count);
    return g;
}
}  // namespace

// C = A B in two passes: a key-only pass counts each row's distinct
// columns (4-byte slots, so four times the warps per SM of the numeric
// pass), then the numeric pass -- binned by that count, so most rows get
// small shared tables -- forms the sums in A's row order, drops
// |v| <= 1e-16 and writes the survivors sorted; rows that lost entries to
// the drop are compacted afterwards.
rb_csr_s* spgemm(const rb_csr_s& A, const rb_csr_s& B) {
    RB_REQUIRE(A.n_cols == B.n_rows, "spgemm: inner dimensions differ");
    const int n = A.n_rows;
    if (n == 0) {
        rb_csr_s* C = new_csr(0, B.n_cols, 0);
        RB_CUDA(cudaMemsetAsync(C->rowptr.get(), 0, sizeof(int), stream()));
        return C;
    }
    // 1. structural counts
    DevArray<int> ub((size_t)n + 1), bins((size_t)3 * n + 3), bcnt(3), scnt((size_t)n + 1);
    bcnt.zero();
    k_spgemm_bound<<<grid_for(n, 256), 256, 0, stream()>>>(n, A.rowptr.get(), A.cols.get(),
                                                          B.rowptr.get(), ub.get(), bins.get(),
                                                          bcnt.get(), kK0 / 2, kK1 / 2);
    RB_CHECK_LAUNCH();
    int hb[3];
    bcnt.download(hb, 3);
    RB_CUDA(cudaStreamSynchronize(stream()));
    if (hb[0]) {
        const size_t sm = (size_t)kKW0 * kK0 * sizeof(int);
        auto kern = k_spgemm_keys<kK0, kKW0>;
        RB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        kern<<<grid_for(hb[0], kKW0), kKW0 * 32, sm, stream()>>>(
            bins.get(), hb[0], A.rowptr.get(), A.cols.get(), B.rowptr.get(), B.cols.get(),
            scnt.get());
        RB_CHECK_LAUNCH();
    }
    if (hb[1]) {
        const size_t sm = (size_t)kKW1 * kK1 * sizeof(int);
        auto kern = k_spgemm_keys<kK1, kKW1>;
        RB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        kern<<<grid_for(hb[1], kKW1), kKW1 * 32, sm, stream()>>>(
            bins.get() + (size_t)n, hb[1], A.rowptr.get(), A.cols.get(), B.rowptr.get(),
            B.cols.get(), scnt.get());
        RB_CHECK_LAUNCH();
    }
    if (hb[2]) {
        GlobalTables g = global_tables(bins.get() + 2 * (size_t)n, hb[2], ub.get(), n);
        DevArray<int> gkeys((size_t)g.total);
        k_spgemm_keys_global<<<grid_for((long)hb[2] * 32, 128), 128, 0, stream()>>>(
            bins.get() + 2 * (size_t)n, hb[2], g.toff.get(), g.tsize.get(), A.rowptr.get(),
            A.cols.get(), B.rowptr.get(), B.cols.get(), gkeys.get(), scnt.get());
        RB_CHECK_LAUNCH();
        RB_CUDA(cudaStreamSynchronize(stream()));
    }
    // 2. capacity layout and numeric pass binned by the structural counts
    DevArray<int> cap((size_t)n + 1);
    const long long capacity = exclusive_scan(scnt.get(), cap.get(), n);
    RB_REQUIRE(capacity <= INT_MAX, "spgemm: product has more than 2^31-1 entries");
    DevArray<int> cols((size_t)std::max<long long>(capacity, 1));
    DevArray<double> vals((size_t)std::max<long long>(capacity, 1));
    bcnt.zero();
    k_bin_rows<<<grid_for(n, 256), 256, 0, stream()>>>(n, scnt.get(), kH0 / 2, kH1 / 2,
                                                       bins.get(), bcnt.get());
    RB_CHECK_LAUNCH();
    bcnt.download(hb, 3);
    RB_CUDA(cudaStreamSynchronize(stream()));
    GlobalTables g = global_tables(bins.get() + 2 * (size_t)n, hb[2], scnt.get(), n);
    DevArray<int> gkeys, glist;
    DevArray<double> gsums;
    if (hb[2]) {
        gkeys.alloc((size_t)g.total);
        gsums.alloc((size_t)g.total);
        glist.alloc((size_t)g.total);
    }
    DevArray<int> cnt((size_t)n + 1);
    std::vector<int> unused;
    spgemm_pass<true>(A, B, bins.get(), hb, unused, g.toff, g.tsize, gkeys, gsums, glist,
                      cnt.get(), cap.get(), cols.get(), vals.get());
    // 3. final layout: the capacity one unless the drop removed entries
    DevArray<int> crp((size_t)n + 1);
    const long long nnz = exclusive_scan(cnt.get(), crp.get(), n);
    rb_csr_s* C = new_csr(n, B.n_cols, 0);
    C->nnz = nnz;
    if (nnz == capacity) {
        C->rowptr = std::move(cap);
        C->cols = std::move(cols);
        C->vals = std::move(vals);
    } else {
        C->rowptr = std::move(crp);
        C->cols.alloc((size_t)std::max<long long>(nnz, 1));
        C->vals.alloc((size_t)std::max<long long>(nnz, 1));
        k_spgemm_compact<<<grid_for(n, 256), 256, 0, stream()>>>(
            n, cap.get(), C->rowptr.get(), cnt.get(), cols.get(), vals.get(), C->cols.get(),
            C->vals.get());
        RB_CHECK_LAUNCH();
    }
    return C;
}

// ParCSRMatrix::mult then mult_T (par_matmult.cpp:73-107, 141-196): AP
// walks A's rows in stored (diagonal-first) order; P^T A P walks the rows of
// R = P^T, which list fine rows in increasing order like the CSC that
// CSR_to_CSC builds.  Then sort + move_diag (par_ruge_stuben_solver.hpp:142-143).
rb_csr_s* rap(const rb_csr_s& A, const rb_csr_s& P, const rb_csr_s* R_in, bool diag_first) {
    RB_REQUIRE(A.n_rows == P.n_rows && A.n_cols == P.n_rows, "rap: A and P do not match");
    rb_csr_s* AP = spgemm(A, P);
    rb_csr_s* Rt = nullptr;
    const rb_csr_s* R = R_in;
    if (!R) { Rt = transpose(P); R = Rt; }
    rb_csr_s* Ac = nullptr;
    try {
        Ac = spgemm(*R, *AP);
    } catch (...) {
        delete AP;
        delete Rt;
        throw;
    }
    delete AP;
    delete Rt;
    if (diag_first) sort_rows_diag_first(*Ac, true);
    return Ac;
}

// ========================================================== colouring ===
// Jones-Plassmann rounds (the multicolour SOR stand-in; not in the
// reference): an uncoloured row that beats every uncoloured neighbour by a
// fixed integer hash (ties by index) takes the smallest colour unused by its
// coloured neighbours.  Rows coloured in a round become visible only to the
// next round, so the colouring does not depend on thread order.
__device__ __forceinline__ unsigned jp_hash(unsigned x) {
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
    return x;
}

__global__ void k_jp_round(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           int* colour, int* left) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int coloured = 0;
    if (i < n && colour[i] < 0) {
        const unsigned hi = jp_hash((unsigned)i);
        bool ok = true;
        for (int j = rp[i]; j < rp[i + 1] && ok; j++) {
            int c = ci[j];
            if (c == i || colour[c] >= 0) continue;
            unsigned hc = jp_hash((unsigned)c);
            if (hc > hi || (hc == hi && c > i)) ok = false;
        }
        if (ok) {
            unsigned long long used = 0;
            for (int j = rp[i]; j < rp[i + 1]; j++) {
                int c = ci[j];
                int cc = colour[c];
                if (c != i && cc >= 0 && cc < 64) used |= 1ull << cc;
            }
            int k = 0;
            while (k < 64 && ((used >> k) & 1ull)) k++;
            colour[i] = -2 - k;   // pending: encoded as -(k+2)
            coloured = 1;
        }
    }
    coloured = __syncthreads_count(coloured);
    if (threadIdx.x == 0 && coloured) atomicAdd(left, coloured);
}

__global__ void k_jp_commit(int n, int* colour, int* maxc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && colour[i] <= -2) {
        colour[i] = -colour[i] - 2;
        atomicMax(maxc, colour[i] + 1);
    }
}

int colour_rows(const rb_csr_s& A, int* colour) {
    const int n = A.n_rows;
    if (n == 0) return 0;
    RB_CUDA(cudaMemsetAsync(colour, 0xff, sizeof(int) * n, stream()));   // -1
    DevArray<int> cntr(2);
    cntr.zero();
    long long done = 0;
    const unsigned g = grid_for(n, 256);
    for (int round = 0; round < 100000 && done < n; round++) {
        RB_CUDA(cudaMemsetAsync(cntr.get(), 0, sizeof(int), stream()));
        k_jp_round<<<g, 256, 0, stream()>>>(n, A.rowptr.get(), A.cols.get(), colour, cntr.get());
        k_jp_commit<<<g, 256, 0, stream()>>>(n, colour, cntr.get() + 1);
        RB_CHECK_LAUNCH();
        done += read_scalar(cntr.get());
    }
    RB_REQUIRE(done == n, "colouring did not terminate");
    return read_scalar(cntr.get() + 1);
}

}  // namespace rb
