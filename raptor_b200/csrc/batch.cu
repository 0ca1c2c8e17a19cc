// batch.cu -- an uneven batch of independent systems through one V-cycle.
//
// Each system gets its own hierarchy, set up exactly as a standalone
// rb_amg_setup would (same glibc weights, same coarsening, same stopping
// size), so the batch changes nothing a system computes.  The levels are
// then packed: level l of the batch is the block-diagonal matrix of level l
// of every system that has one, P_l and R_l likewise (a system whose
// coarsest level is l contributes empty rows to P_l).  One V-cycle of the
// batch is then one ordinary cycle over the packed levels -- one launch per
// operation for all systems together -- plus, at each level, a batched dense
// solve for the systems whose coarsest level it is.  The outer CG keeps
// per-system scalars through segmented reductions, and a whole iteration of
// the batch is replayed from one CUDA graph.  The reference has no batch
// solver; each system here follows its ParMultilevel / PCG semantics.
#include <algorithm>
#include <climits>
#include <cmath>
#include <functional>
#include <memory>
#include <string>

#include "blas1.cuh"
#include "hierarchy.cuh"

namespace rb {

namespace {

constexpr int kSegChunk = 16384;   // rows per reduction chunk (chunks never span systems)

struct SegScal {
    double* rz;
    double* pAp;
    double* alpha;
    double* beta;
    double* rr;
    double* tmp;
    int* active;
    int* breakdown;
};

// Scatter one system's CSR into the packed block-diagonal matrix.
__global__ void k_pack_rows(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                            const double* __restrict__ cv, long row0, long nnz0, long col0,
                            int* prp, int* pci, double* pcv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    prp[row0 + i] = (int)(nnz0 + rp[i]);
    for (int j = rp[i]; j < rp[i + 1]; j++) {
        pci[nnz0 + j] = (int)(col0 + ci[j]);
        pcv[nnz0 + j] = cv[j];
    }
}

__global__ void k_fill_rowptr(int n, long row0, int value, int* prp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) prp[row0 + i] = value;
}

// Dense solve of each listed system's coarsest level (one CTA per system).
// sys / active (optional): a listed system that has stopped is skipped.
template <typename T>
__global__ void k_lu_solve_batch(const int* __restrict__ row0, const int* __restrict__ nrow,
                                 const long long* __restrict__ luo, const int* __restrict__ pivo,
                                 const double* __restrict__ lu_all, const int* __restrict__ piv_all,
                                 const T* __restrict__ b, T* __restrict__ x,
                                 const int* __restrict__ sys, const int* __restrict__ active) {
    if (active && !active[sys[blockIdx.x]]) return;
    extern __shared__ double y[];
    const int n = nrow[blockIdx.x];
    const long r0 = row0[blockIdx.x];
    const double* lu = lu_all + luo[blockIdx.x];
    const int* piv = piv_all + pivo[blockIdx.x];
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = (double)b[r0 + i];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int q = 0; q < n; q++) {
            const int p = piv[q];
            if (p != q) { double t = y[q]; y[q] = y[p]; y[p] = t; }
        }
    __syncthreads();
    for (int j = 0; j < n; j++) {
        const double yj = y[j];
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) y[i] -= lu[i + (size_t)j * n] * yj;
        __syncthreads();
    }
    for (int j = n - 1; j >= 0; j--) {
        if (threadIdx.x == 0) y[j] /= lu[j + (size_t)j * n];
        __syncthreads();
        const double yj = y[j];
        for (int i = threadIdx.x; i < j; i += blockDim.x) y[i] -= lu[i + (size_t)j * n] * yj;
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[r0 + i] = (T)y[i];
}

// x = inv b for each listed system's coarsest level (one CTA per system;
// inverses column-major)
template <typename T>
__global__ void k_coarse_mv_batch(const int* __restrict__ row0, const int* __restrict__ nrow,
                                  const long long* __restrict__ ioff, const double* __restrict__ inv_all,
                                  const T* __restrict__ b, T* __restrict__ x,
                                  const int* __restrict__ sys, const int* __restrict__ active) {
    if (active && !active[sys[blockIdx.x]]) return;
    extern __shared__ double bs[];
    const int n = nrow[blockIdx.x];
    const long r0 = row0[blockIdx.x];
    const double* inv = inv_all + ioff[blockIdx.x];
    for (int i = threadIdx.x; i < n; i += blockDim.x) bs[i] = (double)b[r0 + i];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < n; j++) s += inv[(size_t)j * n + i] * bs[j];
        x[r0 + i] = (T)s;
    }
}

// Segmented dot: one CTA per chunk writes its partial; then one thread per
// system sums that system's chunks in order.  Deterministic.
// gate (optional): the pass runs only when *gate is nonzero (a step of the
// device-side loop that some iterations skip)
// csys / active (optional): a chunk of a stopped system writes 0 unread.
__global__ void __launch_bounds__(256)
k_seg_partial(const int* __restrict__ lo, const int* __restrict__ hi, const double* __restrict__ a,
              const double* __restrict__ b, double* part, const int* gate,
              const int* __restrict__ csys, const int* __restrict__ active) {
    if (gate && *(volatile const int*)gate == 0) return;
    __shared__ double w[8];
    const int c = blockIdx.x;
    if (active && !active[csys[c]]) {
        if (threadIdx.x == 0) part[c] = 0.0;
        return;
    }
    double t = 0.0;
    for (int i = lo[c] + threadIdx.x; i < hi[c]; i += blockDim.x) t += a[i] * b[i];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < 8; k++) s += w[k];
        part[c] = s;
    }
}

template <class Fin>
__global__ void k_seg_finish(int n_sys, const int* __restrict__ chunk0, const double* __restrict__ part,
                             Fin fin, const int* gate) {
    if (gate && *(volatile const int*)gate == 0) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_sys) return;
    double t = 0.0;
    for (int c = chunk0[s]; c < chunk0[s + 1]; c++) t += part[c];
    fin(s, t);
}

struct FinSPAp {
    SegScal S;
    __device__ void operator()(int s, double t) const {
        S.pAp[s] = t;
        if (S.active[s]) {
            S.alpha[s] = S.rz[s] / t;
            if (!(t > 0.0) || !isfinite(t)) *S.breakdown = 1;
        } else {
            S.alpha[s] = 0.0;
        }
    }
};
struct FinSRZ {
    SegScal S;
    __device__ void operator()(int s, double t) const {
        S.beta[s] = (S.active[s] && S.rz[s] != 0.0) ? t / S.rz[s] : 0.0;
        S.rz[s] = t;
    }
};
struct FinSSetRZ {
    SegScal S;
    __device__ void operator()(int s, double t) const { S.rz[s] = t; }
};
struct FinSRR {
    SegScal S;
    __device__ void operator()(int s, double t) const { S.rr[s] = t; }
};
struct FinSTmp {
    SegScal S;
    __device__ void operator()(int s, double t) const { S.tmp[s] = t; }
};

// active (optional): rows of stopped systems are left as they are (their
// alpha and beta are 0, so the update would not change x or r either)
__global__ void k_seg_update(long n, const int* __restrict__ seg, double* __restrict__ x,
                             double* __restrict__ r, const double* __restrict__ p,
                             const double* __restrict__ Ap, const double* __restrict__ alpha,
                             const int* __restrict__ active) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (active && !active[seg[i]]) return;
    const double a = alpha[seg[i]];
    x[i] += p[i] * a;
    r[i] = r[i] + Ap[i] * (-1.0 * a);
}

__global__ void k_seg_p(long n, const int* __restrict__ seg, double* __restrict__ p,
                        const double* __restrict__ z, const double* __restrict__ beta,
                        const int* __restrict__ active) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (active && !active[seg[i]])) return;
    p[i] = p[i] * beta[seg[i]] + z[i];
}

// The row gates of the packed levels: closed[c] = 1 when every system with
// rows in [c 256, (c + 1) 256) of the level has stopped.  Flat over the
// levels (level l owns chunks cbase[l] .. cbase[l + 1] - 1; offs holds the
// level's n_sys + 1 row offsets at l (n_sys + 1)).
__global__ void k_gate_refresh(int L, int n_sys, const long long* __restrict__ offs,
                               const long long* __restrict__ cbase,
                               const int* __restrict__ active, unsigned char* __restrict__ closed) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cbase[L]) return;
    int l = 0;
    while (c >= cbase[l + 1]) l++;
    const long long* off = offs + (size_t)l * (n_sys + 1);
    const long long r0 = (c - cbase[l]) << kGateShift;
    const long long r1 = min(r0 + (1LL << kGateShift), off[n_sys]);
    // the last system whose first row is at or before r0
    int lo = 0, hi = n_sys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= r0) lo = mid;
        else hi = mid - 1;
    }
    unsigned char shut = 1;
    for (int q = lo; q < n_sys && off[q] < r1; q++)
        if (off[q + 1] > r0 && active[q]) {
            shut = 0;
            break;
        }
    closed[c] = shut;
}

template <typename TO, typename TI>
__global__ void k_convert_gated(long n, const TI* __restrict__ in, TO* __restrict__ out,
                                const unsigned char* __restrict__ closed) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !closed[i >> kGateShift]) out[i] = (TO)in[i];
}

// x = dinv .* b (k_scale_first) on the open rows
template <typename T>
__global__ void k_scale_first_gated(long n, const T* __restrict__ b, const T* __restrict__ dinv,
                                    T* __restrict__ x, const unsigned char* __restrict__ closed) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !closed[i >> kGateShift]) x[i] = (T)(b[i] * dinv[i]);
}

// e, restricted to the open rows when Gt
template <bool Gt, class Epi>
auto gated(const Epi& e, const unsigned char* closed) {
    if constexpr (Gt) return row_gate(e, closed);
    else return e;
}

__global__ void k_seg_ids(int n_sys, const long long* __restrict__ off, int* seg) {
    const int s = blockIdx.y;
    if (s >= n_sys) return;
    const long long lo = off[s], hi = off[s + 1];
    for (long long i = lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < hi;
         i += (long long)gridDim.x * blockDim.x)
        seg[i] = s;
}

// State of the device-side PCG loop of a batch (one copy on the device,
// staged through pinned host memory between launches).
struct BatchCtl {
    int it;        // iterations done
    int end;       // the iteration limit
    int pmode;     // 0: p = z already (first iteration, after a restart)
    int full;      // the iteration under way replaces r by b - A x (every 10th)
    int confirm;   // a system's recursive residual met the tolerance
    int restart;   // a candidate failed the true-residual check
    int done;      // every system has stopped
    int pad;
    double tol;
};

__global__ void k_seg_p_dev(long n, const int* __restrict__ seg, double* __restrict__ p,
                            const double* __restrict__ z, const double* __restrict__ beta,
                            const BatchCtl* c, const int* __restrict__ active) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || c->pmode == 0 || !active[seg[i]]) return;
    p[i] = p[i] * beta[seg[i]] + z[i];
}

// active systems whose recursive residual meets the tolerance
__global__ void k_batch_candidates(int n_sys, SegScal S, const double* __restrict__ bnorm,
                                   int* __restrict__ cand, BatchCtl* c) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_sys) return;
    const int cd = S.active[s] && sqrt(S.rr[s]) <= c->tol * bnorm[s];
    cand[s] = cd;
    if (cd) atomicOr(&c->confirm, 1);
}

// a candidate whose true residual (S.tmp) meets the tolerance stops; one
// that does not sends the loop back to the host for a restart
__global__ void k_batch_confirm(int n_sys, SegScal S, const double* __restrict__ bnorm,
                                int* __restrict__ cand, int* __restrict__ iters,
                                double* __restrict__ relres, BatchCtl* c) {
    if (*(volatile const int*)&c->confirm == 0) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_sys || !cand[s]) return;
    cand[s] = 0;
    const double tr = sqrt(S.tmp[s]);
    if (tr <= c->tol * bnorm[s]) {
        S.active[s] = 0;
        iters[s] = c->it + 1;
        relres[s] = tr / bnorm[s];
    } else {
        c->restart = 1;
    }
}

// end of one iteration: count it, set up the next, and end the graph's
// while loop on breakdown, when every system has stopped, on a failed
// confirmation (the host restarts), or at the iteration limit
constexpr int kStepEndThreads = 256;
__global__ void __launch_bounds__(kStepEndThreads)
k_batch_step_end(int n_sys, SegScal S, BatchCtl* c, cudaGraphConditionalHandle h) {
    int any = 0;
    for (int s = threadIdx.x; s < n_sys; s += blockDim.x) any |= S.active[s];
    any = __syncthreads_or(any);
    if (threadIdx.x != 0) return;
    const int it = c->it + 1;
    c->it = it;
    c->pmode = 1;
    c->confirm = 0;
    c->full = ((it + 1) % 10 == 0) ? 1 : 0;
    c->done = any ? 0 : 1;
    const bool stop = *S.breakdown != 0 || !any || c->restart != 0 || it >= c->end;
    cudaGraphSetConditional(h, stop ? 0u : 1u);
}

}  // namespace

struct Batch {
    int n_sys = 0;
    rb_amg_opts opts{};
    std::vector<int> depth;                       // levels of each system
    std::vector<std::vector<long long>> off;      // off[l][s], n_sys + 1 entries
    Hierarchy cat;                                // packed levels
    // coarsest-level LUs
    DevArray<double> lu, inv;   // inv: coarse inverses when every coarsest level is small
    DevArray<int> piv;
    struct CoarseTab {
        int count = 0, max_n = 0;
        DevArray<int> row0, n, pivo, sys;
        DevArray<long long> luo;
    };
    std::vector<CoarseTab> coarse;
    // outer CG
    DevArray<int> seg, chunk_lo, chunk_hi, chunk0;
    int n_chunks = 0;
    DevArray<double> part, r, z, p, Ap, rt;
    DevArray<double> sc;     // 6 n_sys scalars
    DevArray<int> si;        // n_sys active flags + breakdown
    SegScal S{};
    std::vector<double> h_rr, h_tmp;
    std::vector<int> h_active;
    // device-side loop: its state, per-system norms, candidates and results
    DevArray<BatchCtl> ctl;
    BatchCtl* h_ctl = nullptr;
    DevArray<double> bnorm_d, relres_d;
    DevArray<int> cand_d, iters_d;
    int host_waits = 0;   // host waits of the last pcg (one per graph launch)
    // Row gates of the packed levels (one byte per 256 rows, kGateShift):
    // inside pcg every operation of the cycle and of the outer iteration
    // passes over the rows of systems that have stopped, so an iteration
    // costs the rows of the systems still running, not of all of them.
    // Systems are independent (every packed operator is block-diagonal), so
    // a skipped row changes no other system's result.
    DevArray<unsigned char> gates;
    std::vector<long long> gate_base;   // first byte of each level
    DevArray<long long> gate_offs, gate_cbase;
    DevArray<int> chunk_sys;            // system of each reduction chunk
    bool gating = false;                // set while pcg builds its launches
    const unsigned char* gate(int l) const { return gates.get() + gate_base[l]; }
    void refresh_gates() {
        const long long total = gate_base.back();
        if (!total) return;
        k_gate_refresh<<<grid_for(total, 256), 256, 0, stream()>>>(
            (int)off.size(), n_sys, gate_offs.get(), gate_cbase.get(), S.active, gates.get());
        RB_CHECK_LAUNCH();
    }
    ~Batch() {
        if (h_ctl) cudaFreeHost(h_ctl);
    }

    long long rows() const { return off[0][n_sys]; }

    // skip_stopped: chunks of systems that have stopped contribute 0
    template <class Fin>
    void seg_dot(const double* a, const double* b, Fin fin, const int* gate = nullptr,
                 bool skip_stopped = true) {
        k_seg_partial<<<n_chunks, 256, 0, stream()>>>(chunk_lo.get(), chunk_hi.get(), a, b,
                                                      part.get(), gate, chunk_sys.get(),
                                                      gating && skip_stopped ? S.active : nullptr);
        RB_CHECK_LAUNCH();
        k_seg_finish<<<grid_for(n_sys, 128), 128, 0, stream()>>>(n_sys, chunk0.get(), part.get(),
                                                                  fin, gate);
        RB_CHECK_LAUNCH();
    }

    template <typename T>
    void coarse_solve(int l, const T* b, T* x) {
        CoarseTab& t = coarse[l];
        if (!t.count) return;
        const int* act = gating ? S.active : nullptr;
        if (inv.get())
            k_coarse_mv_batch<T><<<t.count, 256, sizeof(double) * std::max(t.max_n, 1), stream()>>>(
                t.row0.get(), t.n.get(), t.luo.get(), inv.get(), b, x, t.sys.get(), act);
        else
            k_lu_solve_batch<T><<<t.count, 256, sizeof(double) * std::max(t.max_n, 1), stream()>>>(
                t.row0.get(), t.n.get(), t.luo.get(), t.pivo.get(), lu.get(), piv.get(), b, x,
                t.sys.get(), act);
        RB_CHECK_LAUNCH();
    }

    void setup(int n, const rb_csr_s* const* mats, const rb_amg_opts& o);
    template <bool Gt, typename T>
    void cycle_level(std::vector<Level<T>>& lv, int l, T* x, const T* b, bool x_zero);
    void cycle64(double* x, const double* b);
    int pcg(double* x, const double* b, double tol, int max_iter, int* iters, double* relres);
    int pcg_device_loop(double* x, const double* b, double tol, int max_iter, int* iters,
                        double* relres, const std::vector<double>& bnorm,
                        const std::function<void()>& restart);
};

void Batch::setup(int n, const rb_csr_s* const* mats, const rb_amg_opts& o) {
    RB_REQUIRE(n >= 1 && n <= 65535, "batch: the number of systems must be in 1..65535");
    n_sys = n;
    opts = o;
    RB_REQUIRE(o.num_smooth_sweeps >= 0, "num_smooth_sweeps < 0");
    // standalone hierarchies (FP64 levels only)
    std::vector<std::unique_ptr<Hierarchy>> sys(n);
    int Lmax = 0;
    depth.assign(n, 0);
    for (int s = 0; s < n; s++) {
        RB_REQUIRE(mats[s] && mats[s]->n_rows == mats[s]->n_cols, "batch: every matrix must be square");
        sys[s].reset(new Hierarchy());
        sys[s]->setup(*mats[s], o, nullptr, false);
        depth[s] = sys[s]->num_levels();
        Lmax = std::max(Lmax, depth[s]);
    }
    // row offsets per level (absent systems have no rows)
    off.assign(Lmax, std::vector<long long>(n + 1, 0));
    for (int l = 0; l < Lmax; l++)
        for (int s = 0; s < n; s++)
            off[l][s + 1] = off[l][s] + (l < depth[s] ? sys[s]->master[l].A->n_rows : 0);
    RB_REQUIRE(off[0][n] <= INT_MAX, "batch: more than 2^31-1 rows in total");
    // pack A_l and P_l block-diagonally
    cat.opts = o;
    cat.use_graphs = o.use_graphs != 0;
    cat.master.clear();
    cat.master.resize(Lmax);
    for (int l = 0; l < Lmax; l++) {
        long long nnzA = 0, nnzP = 0;
        for (int s = 0; s < n; s++) {
            if (l >= depth[s]) continue;
            nnzA += sys[s]->master[l].A->nnz;
            if (l < depth[s] - 1) nnzP += sys[s]->master[l].P->nnz;
        }
        const int rows = (int)off[l][n];
        rb_csr_s* A = new_csr(rows, rows, nnzA);
        cat.master[l].A.reset(A);
        rb_csr_s* P = nullptr;
        if (l < Lmax - 1) {
            P = new_csr(rows, (int)off[l + 1][n], nnzP);
            cat.master[l].P.reset(P);
        }
        long long za = 0, zp = 0;
        for (int s = 0; s < n; s++) {
            if (l >= depth[s]) continue;
            const rb_csr_s& As = *sys[s]->master[l].A;
            const int ns = As.n_rows;
            if (ns)
                k_pack_rows<<<grid_for(ns, 128), 128, 0, stream()>>>(
                    ns, As.rowptr.get(), As.cols.get(), As.vals.get(), off[l][s], za, off[l][s],
                    A->rowptr.get(), A->cols.get(), A->vals.get());
            RB_CHECK_LAUNCH();
            za += As.nnz;
            if (P) {
                if (l < depth[s] - 1) {
                    const rb_csr_s& Ps = *sys[s]->master[l].P;
                    k_pack_rows<<<grid_for(ns, 128), 128, 0, stream()>>>(
                        ns, Ps.rowptr.get(), Ps.cols.get(), Ps.vals.get(), off[l][s], zp,
                        off[l + 1][s], P->rowptr.get(), P->cols.get(), P->vals.get());
                    RB_CHECK_LAUNCH();
                    zp += Ps.nnz;
                } else if (ns) {
                    // coarsest at l: empty rows of P
                    k_fill_rowptr<<<grid_for(ns, 128), 128, 0, stream()>>>(ns, off[l][s], (int)zp,
                                                                           P->rowptr.get());
                    RB_CHECK_LAUNCH();
                }
            }
        }
        const int za_i = (int)za;
        RB_CUDA(cudaMemcpyAsync(A->rowptr.get() + rows, &za_i, sizeof(int), cudaMemcpyHostToDevice,
                                stream()));
        if (P) {
            const int zp_i = (int)zp;
            RB_CUDA(cudaMemcpyAsync(P->rowptr.get() + rows, &zp_i, sizeof(int),
                                    cudaMemcpyHostToDevice, stream()));
            RB_CUDA(cudaStreamSynchronize(stream()));
            cat.master[l].R.reset(transpose(*P));
        }
        RB_CUDA(cudaStreamSynchronize(stream()));
    }
    // coarsest-level LUs (A_c^T, as the standalone hierarchy factors it)
    std::vector<long long> luo(n), pivo(n);
    long long lu_tot = 0, piv_tot = 0;
    for (int s = 0; s < n; s++) {
        const int nc = sys[s]->master[depth[s] - 1].A->n_rows;
        RB_REQUIRE(nc <= 6000, "batch: a coarsest level is too large for the dense solve");
        luo[s] = lu_tot;
        pivo[s] = piv_tot;
        lu_tot += (long long)nc * nc;
        piv_tot += nc;
    }
    lu.alloc((size_t)std::max(lu_tot, 1LL));
    piv.alloc((size_t)std::max(piv_tot, 1LL));
    lu.zero();
    DevArray<int> info(1);
    info.zero();
    for (int s = 0; s < n; s++) {
        const rb_csr_s& Ac = *sys[s]->master[depth[s] - 1].A;
        const int nc = Ac.n_rows;
        if (!nc) continue;
        k_dense_from_csr<<<grid_for(nc, 128), 128, 0, stream()>>>(
            nc, Ac.rowptr.get(), Ac.cols.get(), Ac.vals.get(), lu.get() + luo[s]);
        RB_CHECK_LAUNCH();
        k_lu_factor<<<1, 256, 0, stream()>>>(nc, lu.get() + luo[s], piv.get() + pivo[s], info.get());
        RB_CHECK_LAUNCH();
    }
    int nc_max = 0;
    for (int s = 0; s < n; s++) nc_max = std::max(nc_max, sys[s]->master[depth[s] - 1].A->n_rows);
    if (nc_max <= kCoarseInvMax) {
        inv.alloc((size_t)std::max(lu_tot, 1LL));
        for (int s = 0; s < n; s++) {
            const int nc = sys[s]->master[depth[s] - 1].A->n_rows;
            if (!nc) continue;
            k_lu_invert<<<1, 256, sizeof(double) * nc, stream()>>>(nc, lu.get() + luo[s],
                                                                  piv.get() + pivo[s],
                                                                  inv.get() + luo[s]);
            RB_CHECK_LAUNCH();
        }
    }
    coarse.clear();
    coarse.resize(Lmax);
    for (int l = 0; l < Lmax; l++) {
        std::vector<int> r0, nr, pv, sy;
        std::vector<long long> lo;
        int mx = 0;
        for (int s = 0; s < n; s++) {
            if (depth[s] - 1 != l) continue;
            const int nc = (int)(off[l][s + 1] - off[l][s]);
            if (!nc) continue;
            sy.push_back(s);
            r0.push_back((int)off[l][s]);
            nr.push_back(nc);
            lo.push_back(luo[s]);
            pv.push_back((int)pivo[s]);
            mx = std::max(mx, nc);
        }
        CoarseTab& t = coarse[l];
        t.count = (int)r0.size();
        t.max_n = mx;
        if (t.count) {
            t.row0.alloc(t.count); t.row0.upload(r0.data(), t.count);
            t.n.alloc(t.count); t.n.upload(nr.data(), t.count);
            t.luo.alloc(t.count); t.luo.upload(lo.data(), t.count);
            t.pivo.alloc(t.count); t.pivo.upload(pv.data(), t.count);
            t.sys.alloc(t.count); t.sys.upload(sy.data(), t.count);
        }
    }
    RB_CUDA(cudaStreamSynchronize(stream()));
    sys.clear();
    // cycle data of the packed levels (value copies, inverse diagonals,
    // colourings, kernel widths)
    cat.strided_only = true;
    if (o.precision == RB_PREC_FP32) cat.build_levels(cat.lv32);
    else cat.build_levels(cat.lv64);
    auto zero_levels = [](auto& lv) {
        for (auto& V : lv) {
            V.x.zero();
            V.b.zero();
            V.r.zero();
            V.xt.zero();
        }
    };
    if (o.precision == RB_PREC_FP32) zero_levels(cat.lv32);
    else zero_levels(cat.lv64);
    // row gates: one byte per 256 rows of every packed level
    gate_base.assign(Lmax + 1, 0);
    for (int l = 0; l < Lmax; l++)
        gate_base[l + 1] = gate_base[l] + ((off[l][n] + (1 << kGateShift) - 1) >> kGateShift);
    gates.alloc((size_t)std::max<long long>(gate_base[Lmax], 1));
    gates.zero();
    {
        std::vector<long long> flat;
        for (int l = 0; l < Lmax; l++) flat.insert(flat.end(), off[l].begin(), off[l].end());
        gate_offs.alloc(flat.size());
        gate_offs.upload(flat.data(), flat.size());
        gate_cbase.alloc(gate_base.size());
        gate_cbase.upload(gate_base.data(), gate_base.size());
    }
    // outer CG: segments and chunks of the finest level
    const long long N = off[0][n];
    std::vector<int> clo, chi, c0(n + 1, 0);
    for (int s = 0; s < n; s++) {
        c0[s] = (int)clo.size();
        for (long long a = off[0][s]; a < off[0][s + 1]; a += kSegChunk) {
            clo.push_back((int)a);
            chi.push_back((int)std::min(off[0][s + 1], a + kSegChunk));
        }
    }
    c0[n] = (int)clo.size();
    n_chunks = std::max((int)clo.size(), 1);
    if (clo.empty()) { clo.push_back(0); chi.push_back(0); }
    chunk_lo.alloc(clo.size()); chunk_lo.upload(clo.data(), clo.size());
    chunk_hi.alloc(chi.size()); chunk_hi.upload(chi.data(), chi.size());
    chunk0.alloc(c0.size()); chunk0.upload(c0.data(), c0.size());
    {
        std::vector<int> cs(std::max<size_t>(clo.size(), 1), 0);
        for (int s = 0; s < n; s++)
            for (int c = c0[s]; c < c0[s + 1]; c++) cs[c] = s;
        chunk_sys.alloc(cs.size());
        chunk_sys.upload(cs.data(), cs.size());
    }
    part.alloc((size_t)n_chunks);
    seg.alloc((size_t)std::max<long long>(N, 1));
    DevArray<long long> offd((size_t)n + 1);
    offd.upload(off[0].data(), n + 1);
    k_seg_ids<<<dim3(64, n), 256, 0, stream()>>>(n, offd.get(), seg.get());
    RB_CHECK_LAUNCH();
    const size_t m = (size_t)std::max<long long>(N, 1);
    r.alloc(m); z.alloc(m); p.alloc(m); Ap.alloc(m); rt.alloc(m);
    r.zero(); z.zero(); p.zero(); Ap.zero(); rt.zero();
    sc.alloc((size_t)6 * n);
    si.alloc((size_t)n + 1);
    S = SegScal{sc.get(), sc.get() + n, sc.get() + 2 * n, sc.get() + 3 * n, sc.get() + 4 * n,
                sc.get() + 5 * n, si.get(), si.get() + n};
    h_rr.resize(n);
    h_tmp.resize(n);
    h_active.resize(n);
    RB_CUDA(cudaStreamSynchronize(stream()));
}

// ParMultilevel::cycle on the packed levels, plus the dense solve of the
// systems whose coarsest level is l.  Gt: the rows of systems that have
// stopped are passed over (the row gates; Jacobi-type smoothing only, the
// multicolour sweeps run every row).
template <bool Gt, typename T>
void Batch::cycle_level(std::vector<Level<T>>& lv, int l, T* x, const T* b, bool x_zero) {
    const int L = (int)lv.size();
    if (l == L - 1) {
        coarse_solve<T>(l, b, x);
        return;
    }
    Level<T>& V = lv[l];
    Level<T>& C = lv[l + 1];
    const unsigned char* gl = Gt ? gate(l) : nullptr;
    const unsigned char* gc = Gt ? gate(l + 1) : nullptr;
    const int rt = opts.relax_type;
    const bool jt = (rt == RB_RELAX_JACOBI && !opts.jacobi_compat) || rt == RB_RELAX_L1JACOBI;
    auto smooth = [&](T*& cur, T*& other, bool xz) {
        if (!Gt || !jt || opts.num_smooth_sweeps <= 0) {
            cat.smooth(V, cur, other, b, xz);
            return;
        }
        // Hierarchy::smooth's Jacobi-type sweeps on the open rows
        for (int s = 0; s < opts.num_smooth_sweeps; s++) {
            if (s == 0 && xz) {
                k_scale_first_gated<T><<<grid_for(V.n, 256), 256, 0, stream()>>>(
                    V.n, b, V.dinv.get(), cur, gl);
                RB_CHECK_LAUNCH();
                continue;
            }
            V.apply_A(cur, gated<Gt>(EpiJacobi<T, T, T>{cur, b, V.dinv.get(), other}, gl));
            std::swap(cur, other);
        }
    };
    T* cur = x;
    T* other = V.xt.get();
    smooth(cur, other, x_zero);
    V.apply_A(cur, gated<Gt>(EpiResidual<T, T>{b, V.r.get()}, gl));
    rows_op(V.R, V.R16, C.n, V.r.get(), gated<Gt>(EpiStore<T>{C.b.get()}, gc), V.gR);
    cycle_level<Gt>(lv, l + 1, C.x.get(), C.b.get(), true);
    T* start = x;
    if (jt && (opts.num_smooth_sweeps & 1)) start = (x == V.xt.get()) ? x : V.xt.get();
    if (cur == start) {
        rows_op(V.P, V.P16, V.n, C.x.get(), gated<Gt>(EpiAppend<T>{cur}, gl), V.gP);
    } else {
        rows_op(V.P, V.P16, V.n, C.x.get(), gated<Gt>(EpiAddTo<T>{cur, start}, gl), V.gP);
        cur = start;
    }
    other = (cur == x) ? V.xt.get() : x;
    smooth(cur, other, false);
    if (cur != x)
        RB_CUDA(cudaMemcpyAsync(x, cur, sizeof(T) * V.n, cudaMemcpyDeviceToDevice, stream()));
    // systems whose hierarchy ends here: the direct solve replaces the sweeps
    coarse_solve<T>(l, b, x);
}

void Batch::cycle64(double* x, const double* b) {
    if (opts.precision == RB_PREC_FP32) {
        Level<float>& V = cat.lv32[0];
        const long n = V.n;
        if (gating) {
            k_convert_gated<float, double><<<grid_for(n, 256), 256, 0, stream()>>>(n, b, V.b.get(),
                                                                                  gate(0));
            RB_CHECK_LAUNCH();
            cycle_level<true>(cat.lv32, 0, V.x.get(), V.b.get(), true);
            k_convert_gated<double, float><<<grid_for(n, 256), 256, 0, stream()>>>(n, V.x.get(), x,
                                                                                  gate(0));
            RB_CHECK_LAUNCH();
            return;
        }
        k_convert<float, double><<<grid_for(n, 256), 256, 0, stream()>>>(n, b, V.b.get());
        RB_CHECK_LAUNCH();
        cycle_level<false>(cat.lv32, 0, V.x.get(), V.b.get(), true);
        k_convert<double, float><<<grid_for(n, 256), 256, 0, stream()>>>(n, V.x.get(), x);
        RB_CHECK_LAUNCH();
    } else if (gating) {
        cycle_level<true>(cat.lv64, 0, x, b, true);
    } else {
        cycle_level<false>(cat.lv64, 0, x, b, true);
    }
}

// Per-system PCG in true-residual mode: recursive residual replaced by
// b - A x every 10 iterations, a system stops once its true relative
// residual meets tol; stopped systems keep alpha = beta = 0.
int Batch::pcg(double* x, const double* b, double tol, int max_iter, int* iters, double* relres) {
    struct GatingOn {
        bool& g;
        explicit GatingOn(bool& f) : g(f) { g = true; }
        ~GatingOn() { g = false; }
    } gating_on(gating);
    const rb_csr_s& A = *cat.master[0].A;
    const long N = A.n_rows;
    const int n = n_sys;
    if (max_iter <= 0) max_iter = 1000;
    const CsrView<double> Av = view(A);
    auto read = [&](std::vector<double>& dst, const double* src) {
        RB_CUDA(cudaMemcpyAsync(dst.data(), src, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                stream()));
        RB_CUDA(cudaStreamSynchronize(stream()));
    };
    auto push_active = [&]() {
        RB_CUDA(cudaMemcpyAsync(S.active, h_active.data(), sizeof(int) * n, cudaMemcpyHostToDevice,
                                stream()));
        refresh_gates();
    };
    RB_CUDA(cudaMemsetAsync(sc.get(), 0, sizeof(double) * 6 * n, stream()));
    RB_CUDA(cudaMemsetAsync(si.get(), 0, sizeof(int) * (n + 1), stream()));
    seg_dot(b, b, FinSTmp{S}, nullptr, false);
    read(h_tmp, S.tmp);
    std::vector<double> bnorm(n);
    for (int s = 0; s < n; s++) {
        bnorm[s] = std::sqrt(h_tmp[s]);
        h_active[s] = bnorm[s] > 0.0 ? 1 : 0;
        iters[s] = 0;
        relres[s] = 0.0;
    }
    push_active();
    auto restart = [&]() {
        residual64(Av, x, b, r.get());
        cycle64(z.get(), r.get());
        RB_CUDA(cudaMemcpyAsync(p.get(), z.get(), sizeof(double) * N, cudaMemcpyDeviceToDevice,
                                stream()));
        seg_dot(r.get(), z.get(), FinSSetRZ{S});
        seg_dot(r.get(), r.get(), FinSRR{S});
    };
    restart();
    read(h_rr, S.rr);
    int iter = 0;
    auto check = [&]() -> bool {
        bool candidate = false;
        for (int s = 0; s < n; s++)
            if (h_active[s] && std::sqrt(h_rr[s]) <= tol * bnorm[s]) candidate = true;
        if (candidate) {
            residual64(Av, x, b, rt.get());
            seg_dot(rt.get(), rt.get(), FinSTmp{S});
            read(h_tmp, S.tmp);
            bool failed = false;
            for (int s = 0; s < n; s++) {
                if (!h_active[s] || std::sqrt(h_rr[s]) > tol * bnorm[s]) continue;
                const double tr = std::sqrt(h_tmp[s]);
                if (tr <= tol * bnorm[s]) {
                    h_active[s] = 0;
                    iters[s] = iter;
                    relres[s] = tr / bnorm[s];
                } else {
                    failed = true;
                }
            }
            push_active();
            if (failed) {
                restart();
                read(h_rr, S.rr);
            }
        }
        for (int s = 0; s < n; s++)
            if (h_active[s]) return false;
        return true;
    };
    if (check()) return RB_OK;
    host_waits = 0;
    if (cat.use_graphs) return pcg_device_loop(x, b, tol, max_iter, iters, relres, bnorm, restart);
    auto body = [&](bool full_r) {
        launch_rows(Av.rowptr, Av.cols, Av.vals, N, Av.nnz, p.get(),
                    row_gate(EpiStore<double>{Ap.get()}, gate(0)), cat.gA0 > 0 ? cat.gA0 : 0);
        seg_dot(p.get(), Ap.get(), FinSPAp{S});
        k_seg_update<<<grid_for(N, 256), 256, 0, stream()>>>(N, seg.get(), x, r.get(), p.get(),
                                                             Ap.get(), S.alpha, S.active);
        RB_CHECK_LAUNCH();
        if (full_r)
            launch_rows(Av.rowptr, Av.cols, Av.vals, N, Av.nnz, x,
                        row_gate(EpiResidual<double, double>{b, r.get()}, gate(0)),
                        cat.gA0 > 0 ? cat.gA0 : 0);
        seg_dot(r.get(), r.get(), FinSRR{S});
        cycle64(z.get(), r.get());
        seg_dot(r.get(), z.get(), FinSRZ{S});
    };
    int status = RB_ERR_NOT_CONVERGED;
    int h_break = 0;
    while (iter < max_iter) {
        iter++;
        const bool full_r = iter % 10 == 0;
        char key[96];
        snprintf(key, sizeof(key), "batch%s:%p:%p", full_r ? "F" : "", (void*)x, (const void*)b);
        cat.run_graph(key, [&] { body(full_r); });
        read(h_rr, S.rr);
        RB_CUDA(cudaMemcpyAsync(&h_break, S.breakdown, sizeof(int), cudaMemcpyDeviceToHost, stream()));
        RB_CUDA(cudaStreamSynchronize(stream()));
        if (h_break) return RB_ERR_BREAKDOWN;
        if (check()) { status = RB_OK; break; }
        k_seg_p<<<grid_for(N, 256), 256, 0, stream()>>>(N, seg.get(), p.get(), z.get(), S.beta,
                                                        S.active);
        RB_CHECK_LAUNCH();
    }
    if (status != RB_OK)
        for (int s = 0; s < n; s++)
            if (h_active[s]) {
                iters[s] = iter;
                relres[s] = std::sqrt(h_rr[s]) / bnorm[s];
            }
    return status;
}

// The iterations of Batch::pcg on the device: one graph launch holds a
// while loop whose body is one iteration for every system (p update, A p and
// alpha, x and r updates, the every-10th b - A x, r.r, the V-cycle and r.z),
// followed by the stopping logic the host loop runs otherwise: systems whose
// recursive residual meets the tolerance are confirmed with the true
// residual (b - A x and its segmented norm, gated to the iterations that
// need them) and stop; the loop ends when all have stopped, on breakdown, at
// the iteration limit, or when a confirmation fails, after which the host
// restarts the recurrence (r = b - A x, z = M r, p = z) exactly as before and
// launches again.  The host therefore waits once per launch, not once per
// iteration; results are the same as the host loop's.
int Batch::pcg_device_loop(double* x, const double* b, double tol, int max_iter, int* iters,
                           double* relres, const std::vector<double>& bnorm,
                           const std::function<void()>& restart) {
    const rb_csr_s& A = *cat.master[0].A;
    const long N = A.n_rows;
    const int n = n_sys;
    const CsrView<double> Av = view(A);
    if (!ctl.get()) {
        ctl.alloc(1);
        bnorm_d.alloc((size_t)n);
        relres_d.alloc((size_t)n);
        cand_d.alloc((size_t)n);
        iters_d.alloc((size_t)n);
        RB_CUDA(cudaMallocHost(&h_ctl, sizeof(BatchCtl)));
    }
    bnorm_d.upload(bnorm.data(), n);
    iters_d.upload(iters, n);
    relres_d.upload(relres, n);
    cand_d.zero();
    *h_ctl = BatchCtl{0, max_iter, 0, 0, 0, 0, 0, 0, tol};
    BatchCtl* C = ctl.get();
    const unsigned sg = grid_for(n, 128);
    auto iteration = [&](cudaGraphConditionalHandle h) {
        k_seg_p_dev<<<grid_for(N, 256), 256, 0, stream()>>>(N, seg.get(), p.get(), z.get(),
                                                            S.beta, C, S.active);
        RB_CHECK_LAUNCH();
        launch_rows(Av.rowptr, Av.cols, Av.vals, N, Av.nnz, p.get(),
                    row_gate(EpiStore<double>{Ap.get()}, gate(0)), cat.gA0 > 0 ? cat.gA0 : 0);
        seg_dot(p.get(), Ap.get(), FinSPAp{S});
        k_seg_update<<<grid_for(N, 256), 256, 0, stream()>>>(N, seg.get(), x, r.get(), p.get(),
                                                             Ap.get(), S.alpha, S.active);
        RB_CHECK_LAUNCH();
        launch_rows(Av.rowptr, Av.cols, Av.vals, N, Av.nnz, x,
                    row_gate(EpiResidualIf<double, double>{b, r.get(), &C->full}, gate(0)),
                    cat.gA0 > 0 ? cat.gA0 : 0);
        seg_dot(r.get(), r.get(), FinSRR{S});
        cycle64(z.get(), r.get());
        seg_dot(r.get(), z.get(), FinSRZ{S});
        k_batch_candidates<<<sg, 128, 0, stream()>>>(n, S, bnorm_d.get(), cand_d.get(), C);
        RB_CHECK_LAUNCH();
        launch_rows(Av.rowptr, Av.cols, Av.vals, N, Av.nnz, x,
                    row_gate(EpiResidualIf<double, double>{b, rt.get(), &C->confirm}, gate(0)),
                    cat.gA0 > 0 ? cat.gA0 : 0);
        seg_dot(rt.get(), rt.get(), FinSTmp{S}, &C->confirm);
        k_batch_confirm<<<sg, 128, 0, stream()>>>(n, S, bnorm_d.get(), cand_d.get(),
                                                  iters_d.get(), relres_d.get(), C);
        RB_CHECK_LAUNCH();
        refresh_gates();
        k_batch_step_end<<<1, kStepEndThreads, 0, stream()>>>(n, S, C, h);
        RB_CHECK_LAUNCH();
    };
    char key[96];
    snprintf(key, sizeof(key), "bloop:%p:%p", (void*)x, (const void*)b);
    int status = RB_ERR_NOT_CONVERGED;
    int h_break = 0;
    for (;;) {
        RB_CUDA(cudaMemcpyAsync(C, h_ctl, sizeof(BatchCtl), cudaMemcpyHostToDevice, stream()));
        const int it0 = h_ctl->it;
        cat.run_while_graph(key, iteration);
        RB_CUDA(cudaMemcpyAsync(h_ctl, C, sizeof(BatchCtl), cudaMemcpyDeviceToHost, stream()));
        RB_CUDA(cudaMemcpyAsync(&h_break, S.breakdown, sizeof(int), cudaMemcpyDeviceToHost,
                                stream()));
        RB_CUDA(cudaStreamSynchronize(stream()));
        host_waits++;
        launch_counter() += cat.graph_kernels[key] * (h_ctl->it - it0);
        if (h_break) return RB_ERR_BREAKDOWN;
        if (h_ctl->done) { status = RB_OK; break; }
        if (h_ctl->restart) {
            // as the host loop: deactivated systems stay stopped, the others
            // restart from their true residual
            restart();
            h_ctl->restart = 0;
            h_ctl->pmode = 0;
        }
        if (h_ctl->it >= max_iter) break;
    }
    const int iter = h_ctl->it;
    iters_d.download(iters, n);
    relres_d.download(relres, n);
    RB_CUDA(cudaMemcpyAsync(h_active.data(), S.active, sizeof(int) * n, cudaMemcpyDeviceToHost,
                            stream()));
    RB_CUDA(cudaMemcpyAsync(h_rr.data(), S.rr, sizeof(double) * n, cudaMemcpyDeviceToHost,
                            stream()));
    RB_CUDA(cudaStreamSynchronize(stream()));
    for (int s = 0; s < n; s++)
        if (h_active[s]) {
            iters[s] = iter;
            relres[s] = std::sqrt(h_rr[s]) / bnorm[s];
        }
    return status;
}

}  // namespace rb

struct rb_batch_s {
    rb::Batch b;
};

namespace rb {

rb_batch_s* batch_setup(int n, const rb_csr_s* const* mats, const rb_amg_opts& o) {
    std::unique_ptr<rb_batch_s> B(new rb_batch_s());
    B->b.setup(n, mats, o);
    return B.release();
}
void batch_destroy(rb_batch_s* B) { delete B; }
int batch_num_systems(const rb_batch_s* B) { return B->b.n_sys; }
long long batch_offset(const rb_batch_s* B, int s) { return B->b.off[0][s]; }
int batch_levels(const rb_batch_s* B, int s) { return B->b.depth[s]; }
int batch_packed_levels(const rb_batch_s* B) { return (int)B->b.off.size(); }
void batch_cycle(rb_batch_s* B, double* x, const double* b) {
    Batch& T = B->b;
    char key[96];
    snprintf(key, sizeof(key), "bcyc:%p:%p", (void*)x, (const void*)b);
    T.cat.run_graph(key, [&] { T.cycle64(x, b); });
}
int batch_host_waits(const rb_batch_s* B) { return B->b.host_waits; }
int batch_pcg(rb_batch_s* B, double* x, const double* b, double tol, int max_iter, int* iters,
              double* relres) {
    return B->b.pcg(x, b, tol, max_iter, iters, relres);
}

}  // namespace rb
