// coarsen_rs.cu -- Ruge-Stuben C/F splitting, on the host.
//
// The first pass of Ruge-Stuben coarsening is a greedy sweep: repeatedly take
// the unassigned point of largest measure (how many points strongly depend
// on it), make it a C point, make its unassigned dependents F points, and
// raise the measure of every unassigned point those new F points depend on
// (lower it for points the new C point depends on).  Each step depends on
// every earlier one, so there is no parallel form that selects the same
// points; like the reference, it runs sequentially (here on the host, over
// the strength matrix copied from the device), and the states go back to the
// device for interpolation.  This follows split_rs / rs_first_pass /
// rs_second_pass (ruge_stuben/cf_splitting.cpp:9-328) step for step: the
// measure buckets are kept in one array ordered by measure, a point whose
// measure changes is swapped to the edge of its bucket and the bucket
// boundary moved, and the sweep visits the array from the top down, so ties
// break exactly as the reference's do.  The parallel entry point at one rank
// (split_rs, par_cf_splitting.cpp:7-30) sets the initial states first
// (set_initial_states, :114-131): a row of S with no entry but its diagonal
// has no neighbours.
#include <algorithm>
#include <vector>

#include "rb_internal.cuh"

namespace rb {

namespace {

constexpr int kSel = 1, kUnsel = 0, kUnassign = -1, kNoNbr = -2;   // core/types.hpp:31-37

// First entry of row i past a leading diagonal.
inline int row_begin(const std::vector<int>& rp, const std::vector<int>& ci, int i) {
    int s = rp[i];
    if (s < rp[i + 1] && ci[s] == i) s++;
    return s;
}

// The measure buckets: pos_col[p] is the point at position p, col_pos its
// inverse; bucket m holds positions [start[m], start[m] + size[m]).
struct Buckets {
    std::vector<int> start, size, pos_col, col_pos;
    void swap_positions(int a, int b) {
        col_pos[pos_col[a]] = b;
        col_pos[pos_col[b]] = a;
        std::swap(pos_col[a], pos_col[b]);
    }
};

void rs_first(int n, const std::vector<int>& rp, const std::vector<int>& ci,
              const std::vector<int>& tp, const std::vector<int>& tci, std::vector<int>& meas,
              std::vector<int>& st) {
    Buckets B;
    B.start.assign((size_t)n + 1, 0);
    B.size.assign((size_t)n, 0);
    B.pos_col.assign((size_t)n, 0);
    B.col_pos.assign((size_t)n, 0);
    for (int i = 0; i < n; i++) B.size[meas[i]]++;
    for (int m = 0; m < n; m++) {
        B.start[m + 1] = B.start[m] + B.size[m];
        B.size[m] = 0;
    }
    for (int i = 0; i < n; i++) {
        const int p = B.start[meas[i]] + B.size[meas[i]]++;
        B.pos_col[p] = i;
        B.col_pos[i] = p;
    }
    for (int top = n - 1; top >= 0; top--) {
        const int c = B.pos_col[top];
        B.size[meas[c]]--;
        if (st[c] != kUnassign) continue;
        st[c] = kSel;
        // c's unassigned dependents become F points; every unassigned point
        // an F point depends on gains one in measure (moved to the end of its
        // bucket, which then belongs to the next bucket)
        for (int j = tp[c]; j < tp[c + 1]; j++) {
            const int f = tci[j];
            if (st[f] != kUnassign) continue;
            st[f] = kUnsel;
            for (int k = row_begin(rp, ci, f); k < rp[f + 1]; k++) {
                const int u = ci[k];
                if (st[u] != kUnassign) continue;
                const int m = meas[u];
                if (m >= n - 1) continue;
                const int to = B.start[m] + B.size[m] - 1;
                B.swap_positions(B.col_pos[u], to);
                B.size[m]--;
                B.size[m + 1]++;
                B.start[m + 1] = to;
                meas[u]++;
            }
        }
        // every unassigned point c depends on loses one (moved to the start
        // of its bucket, which then belongs to the previous bucket)
        for (int k = row_begin(rp, ci, c); k < rp[c + 1]; k++) {
            const int u = ci[k];
            if (st[u] != kUnassign) continue;
            const int m = meas[u];
            if (m == 0) continue;
            B.swap_positions(B.col_pos[u], B.start[m]);
            B.size[m]--;
            B.size[m - 1]++;
            B.start[m]++;
            B.start[m - 1] = B.start[m] - B.size[m - 1];
            meas[u]--;
        }
    }
}

// Second pass: an F point i with a strong F neighbour j that shares none of
// i's C points makes j a C point.
void rs_second(int n, const std::vector<int>& rp, const std::vector<int>& ci,
               std::vector<int>& st) {
    std::vector<int> marker((size_t)n, -1);   // marker[c] = i: c is a C point of row i
    for (int i = 0; i < n; i++) {
        if (st[i] == kSel) continue;
        for (int j = rp[i]; j < rp[i + 1]; j++)
            if (st[ci[j]] == kSel) marker[ci[j]] = i;
        for (int j = rp[i]; j < rp[i + 1]; j++) {
            const int f = ci[j];
            if (st[f] != kUnsel) continue;
            if (rp[f] == rp[f + 1]) continue;
            bool shared = false;
            for (int k = rp[f]; k < rp[f + 1] && !shared; k++) shared = marker[ci[k]] == i;
            if (!shared) {
                marker[f] = i;
                st[f] = kSel;
            }
        }
    }
}

}  // namespace

void split_rs(const rb_csr_s& S, int* states_dev, bool second_pass) {
    const int n = S.n_rows;
    if (n == 0) return;
    std::vector<int> rp((size_t)n + 1), ci((size_t)std::max<long long>(S.nnz, 1));
    S.rowptr.download(rp.data(), (size_t)n + 1);
    if (S.nnz) S.cols.download(ci.data(), (size_t)S.nnz);
    RB_CUDA(cudaStreamSynchronize(stream()));
    std::vector<int> st((size_t)n);
    for (int i = 0; i < n; i++) st[i] = (rp[i + 1] - rp[i] > 1) ? kUnassign : kNoNbr;
    // points that depend on each point (off-diagonal entries of S by column,
    // rows in increasing order), and the initial measures
    std::vector<int> tp((size_t)n + 1, 0), tci;
    for (int i = 0; i < n; i++)
        for (int k = row_begin(rp, ci, i); k < rp[i + 1]; k++) tp[ci[k] + 1]++;
    for (int i = 0; i < n; i++) tp[i + 1] += tp[i];
    tci.assign((size_t)std::max(tp[n], 1), 0);
    {
        std::vector<int> fill(tp.begin(), tp.end() - 1);
        for (int i = 0; i < n; i++)
            for (int k = row_begin(rp, ci, i); k < rp[i + 1]; k++) tci[fill[ci[k]]++] = i;
    }
    std::vector<int> meas((size_t)n);
    for (int i = 0; i < n; i++) meas[i] = tp[i + 1] - tp[i];
    rs_first(n, rp, ci, tp, tci, meas, st);
    if (second_pass) rs_second(n, rp, ci, st);
    RB_CUDA(cudaMemcpyAsync(states_dev, st.data(), sizeof(int) * n, cudaMemcpyHostToDevice,
                            stream()));
    RB_CUDA(cudaStreamSynchronize(stream()));
}

}  // namespace rb
