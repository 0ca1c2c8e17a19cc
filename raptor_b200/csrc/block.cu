// block.cu -- k right-hand sides over one hierarchy (the batching form).
//
// The block V-cycle applies the same preconditioner to k columns in one
// pass per operator: every SpMM reads A_l, P_l, R_l once for all columns.
// The block PCG runs k independent conjugate-gradient recurrences (per-column
// alpha, beta and stopping test, all on the device) that share those passes.
// A column that has converged keeps alpha = beta = 0, so its iterate no
// longer changes while the others continue.  Like RB_PCG_TRUE_RESIDUAL, the
// recursive residual is replaced by b - A x every 10 iterations and a
// column stops only once its true relative residual meets the tolerance.
// The reference has no counterpart: it solves one right-hand side at a time.
#include <algorithm>
#include <cmath>
#include <string>

#include "blas1.cuh"
#include "block.cuh"
#include "hierarchy.cuh"

namespace rb {

struct BlockScal {
    double rz[kMaxBlockK];
    double pAp[kMaxBlockK];
    double alpha[kMaxBlockK];
    double beta[kMaxBlockK];
    double rr[kMaxBlockK];
    double tmp[kMaxBlockK];
    int active[kMaxBlockK];
    int breakdown;
};

template <typename T>
struct BLevel {
    DevArray<T> x, b, r, xt;
    int sA = 1, sP = 1, sR = 1;   // rows split S of the SpMM tile, per operator
};

struct BlockState {
    int k = 0;
    std::vector<BLevel<float>> l32;
    std::vector<BLevel<double>> l64;
    DevArray<double> R, Z, P, AP, Rt;
    DevArray<BlockScal> scal;
    BlockScal* host = nullptr;
    int sA0 = 1;   // tile shape of the caller's FP64 A (true residuals)
    ~BlockState() {
        if (host) cudaFreeHost(host);
    }
};

namespace {

struct FinBPAp {
    BlockScal* s;
    __device__ void operator()(int c, double t) const {
        s->pAp[c] = t;
        if (s->active[c]) {
            s->alpha[c] = s->rz[c] / t;
            if (!(t > 0.0) || !isfinite(t)) s->breakdown = 1;
        } else {
            s->alpha[c] = 0.0;
        }
    }
};
struct FinBRZ {
    BlockScal* s;
    __device__ void operator()(int c, double t) const {
        s->beta[c] = (s->active[c] && s->rz[c] != 0.0) ? t / s->rz[c] : 0.0;
        s->rz[c] = t;
    }
};
struct FinBSetRZ {
    BlockScal* s;
    __device__ void operator()(int c, double t) const { s->rz[c] = t; }
};
struct FinBRR {
    BlockScal* s;
    __device__ void operator()(int c, double t) const { s->rr[c] = t; }
};
struct FinBTmp {
    BlockScal* s;
    __device__ void operator()(int c, double t) const { s->tmp[c] = t; }
};

// X += alpha_c P ; R -= alpha_c AP ; rr_c = R_c . R_c; r32 (optional): R in
// FP32 as well (the next block cycle's right-hand side in the FP32 form)
template <int KP>
__global__ void __launch_bounds__(256)
k_bcg_update(long n, int k, double* __restrict__ X, double* __restrict__ R,
             const double* __restrict__ P, const double* __restrict__ AP,
             const BlockScal* __restrict__ s, ReduceSlot rs, FinBRR fin, float* __restrict__ r32) {
    constexpr int RPW = 32 / KP;
    const int lane = threadIdx.x & 31;
    const int c = lane % KP, sub = lane / KP;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    double t = 0.0;
    if (c < k) {
        const double alpha = s->alpha[c];
        for (long i = gwarp * RPW + sub; i < n; i += nwarps * RPW) {
            const long e = i * k + c;
            X[e] += P[e] * alpha;
            const double ri = R[e] + AP[e] * (-1.0 * alpha);
            R[e] = ri;
            if (r32) r32[e] = (float)ri;
            t += ri * ri;
        }
    }
    block_reduce_cols<KP>(t, k, rs, fin);
}

// P = Z + beta_c P (P = Z on a restart); Z FP64 or the FP32 output of the
// block cycle.  Thread t: row t / KP, column t % KP.
template <int KP, typename TZ>
__global__ void k_bcg_p(long n, int k, double* __restrict__ P, const TZ* __restrict__ Z,
                        const BlockScal* __restrict__ s, int restart) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long i = t / KP;
    const int c = (int)(t % KP);
    if (i >= n || c >= k) return;
    const long e = i * k + c;
    if (restart) P[e] = (double)Z[e];
    else P[e] = P[e] * s->beta[c] + (double)Z[e];
}

std::string bkey(const char* tag, int k, const void* a, const void* b, const void* c) {
    char buf[192];
    snprintf(buf, sizeof(buf), "%s%d:%p:%p:%p", tag, k, a, b, c);
    return buf;
}

bool jacobi_type(const rb_amg_opts& o) {
    return (o.relax_type == RB_RELAX_JACOBI && !o.jacobi_compat) || o.relax_type == RB_RELAX_L1JACOBI;
}

template <typename T, class Epi>
void apply_A_block(const Level<T>& V, const BLevel<T>& W, const T* X, int k, Epi epi) {
    if (V.dia) launch_dia_block(V.off, V.Adia.get(), V.n, k, X, epi);
    else launch_csr_block(V.A.rowptr, V.A.cols, V.A.vals, V.n, k, X, epi, W.sA);
}

// Tile shape of one SpMM: rows split S in {1, 2, 4} (S KP <= 32), timed.
template <typename T>
int tune_split(const CsrView<T>& M, int k, const T* xin, T* yout, const char* op) {
    const int KP = pow2_at_least(k);
    if (M.n_rows < 4096 || KP >= 32) return 1;
    const std::string key = tune_key((std::string(op) + std::to_string(k)).c_str(), M.n_rows,
                                     M.nnz, (int)sizeof(T));
    auto& c = tune_cache();
    auto it = c.m.find(key);
    if (it != c.m.end()) return it->second;
    float best = 1e30f;
    int bestS = 1;
    for (int S = 1; S <= 4 && S * KP <= 32; S <<= 1) {
        const float t = time_launch([&] {
            launch_csr_block(M.rowptr, M.cols, M.vals, M.n_rows, k, xin, BStore<T>{yout}, S);
        }, xin, sizeof(T) * (size_t)M.n_cols * (size_t)k);
        if (t < best) { best = t; bestS = S; }
    }
    c.m[key] = bestS;
    tune_save();
    return bestS;
}

template <typename T>
void build_block_levels(std::vector<Level<T>>& lv, std::vector<BLevel<T>>& bl, int k) {
    const int L = (int)lv.size();
    bl.clear();
    bl.resize(L);
    for (int l = 0; l < L; l++) {
        const size_t m = (size_t)std::max(lv[l].n, 1) * k;
        bl[l].x.alloc(m);
        bl[l].b.alloc(m);
        bl[l].r.alloc(m);
        bl[l].xt.alloc(m);
        bl[l].x.zero();
        bl[l].b.zero();
    }
    for (int l = 0; l < L; l++) {
        Level<T>& V = lv[l];
        BLevel<T>& W = bl[l];
        if (!V.dia) W.sA = tune_split(V.A, k, W.x.get(), W.r.get(), "bA");
        if (l < L - 1) {
            W.sP = tune_split(V.P, k, bl[l + 1].x.get(), W.xt.get(), "bP");
            W.sR = tune_split(V.R, k, W.r.get(), bl[l + 1].b.get(), "bR");
        }
    }
}

template <typename T>
void bsmooth(const Hierarchy& H, const Level<T>& V, const BLevel<T>& W, T*& cur, T*& other,
             const T* b, bool x_zero, int k) {
    const int sweeps = H.opts.num_smooth_sweeps;
    const bool jt = jacobi_type(H.opts);
    if (x_zero && !(jt && sweeps > 0))
        RB_CUDA(cudaMemsetAsync(cur, 0, sizeof(T) * (size_t)V.n * k, stream()));
    if (!jt) return;   // Jacobi in compatibility mode leaves x unchanged
    for (int s = 0; s < sweeps; s++) {
        if (s == 0 && x_zero) {
            if (const int lpr = vec_lanes(k, b, BStore<T>{cur})) {
                RB_BLOCK_LPR_SWITCH(lpr, {
                    k_scale_first_block_v<kL, T><<<grid_for((long)V.n * kL, 256), 256, 0,
                                                   stream()>>>(V.n, k, b, V.dinv.get(), cur);
                });
            } else {
                RB_BLOCK_KP_SWITCH(pow2_at_least(k), {
                    k_scale_first_block<kKP, T><<<grid_for((long)V.n * kKP, 256), 256, 0,
                                                  stream()>>>(V.n, k, b, V.dinv.get(), cur);
                });
            }
            RB_CHECK_LAUNCH();
            continue;
        }
        apply_A_block(V, W, cur, k, BJacobi<T>{cur, b, V.dinv.get(), other});
        std::swap(cur, other);
    }
}

template <typename T>
void block_cycle_level(Hierarchy& H, std::vector<Level<T>>& lv, std::vector<BLevel<T>>& bl, int l,
                       T* X, const T* B, bool x_zero, int k) {
    const int L = (int)lv.size();
    if (l == L - 1) {
        if (H.coarse_n && H.cinv.get())
            k_coarse_mv<T><<<k, 256, sizeof(double) * H.coarse_n, stream()>>>(H.coarse_n,
                                                                              H.cinv.get(), k, B, X);
        else if (H.coarse_n)
            k_lu_solve_block<T><<<k, 256, sizeof(double) * H.coarse_n, stream()>>>(
                H.coarse_n, k, H.lu.get(), H.piv.get(), B, X);
        RB_CHECK_LAUNCH();
        return;
    }
    Level<T>& V = lv[l];
    Level<T>& C = lv[l + 1];
    BLevel<T>& W = bl[l];
    BLevel<T>& WC = bl[l + 1];
    T* cur = X;
    T* other = W.xt.get();
    bsmooth(H, V, W, cur, other, B, x_zero, k);
    apply_A_block(V, W, cur, k, BResidual<T, T>{B, W.r.get()});
    launch_csr_block(V.R.rowptr, V.R.cols, V.R.vals, C.n, k, W.r.get(), BStore<T>{WC.b.get()}, W.sR);
    block_cycle_level(H, lv, bl, l + 1, WC.x.get(), WC.b.get(), true, k);
    // x += P x_c into the buffer from which the post-smoothing ping-pong ends in X
    T* start = X;
    if (jacobi_type(H.opts) && (H.opts.num_smooth_sweeps & 1))
        start = (X == W.xt.get()) ? X : W.xt.get();
    if (cur == start) {
        launch_csr_block(V.P.rowptr, V.P.cols, V.P.vals, V.n, k, WC.x.get(), BAppend<T>{cur}, W.sP);
    } else {
        launch_csr_block(V.P.rowptr, V.P.cols, V.P.vals, V.n, k, WC.x.get(),
                         BAddTo<T>{cur, start}, W.sP);
        cur = start;
    }
    other = (cur == X) ? W.xt.get() : X;
    bsmooth(H, V, W, cur, other, B, false, k);
    if (cur != X)
        RB_CUDA(cudaMemcpyAsync(X, cur, sizeof(T) * (size_t)V.n * k, cudaMemcpyDeviceToDevice,
                                stream()));
}

// Z = M R on FP64 blocks of the finest size (conversions at the edges of
// an FP32 hierarchy).
void block_cycle64(Hierarchy& H, BlockState& bs, double* Z, const double* R) {
    const int k = bs.k;
    if (H.opts.precision == RB_PREC_FP32) {
        const long m = (long)H.lv32[0].n * k;
        float* bb = bs.l32[0].b.get();
        float* xx = bs.l32[0].x.get();
        k_convert<float, double><<<grid_for(m, 256), 256, 0, stream()>>>(m, R, bb);
        RB_CHECK_LAUNCH();
        block_cycle_level(H, H.lv32, bs.l32, 0, xx, bb, true, k);
        k_convert<double, float><<<grid_for(m, 256), 256, 0, stream()>>>(m, xx, Z);
        RB_CHECK_LAUNCH();
    } else {
        block_cycle_level(H, H.lv64, bs.l64, 0, Z, R, true, k);
    }
}

// AP = A P with p.Ap per column: the FP32 copy of A_0 (FP64 accumulation)
// in the FP32 form when A is the setup matrix, else the FP64 operator.
void block_outer_apply(Hierarchy& H, BlockState& bs, const rb_csr_s& A, const double* P,
                       double* AP) {
    const long n = A.n_rows;
    const int k = bs.k;
    FinBPAp fin{bs.scal.get()};
    if (H.is_finest(A) && H.opts.precision == RB_PREC_FP32) {
        const Level<float>& V = H.lv32[0];
        if (V.dia) launch_dia_block_dot(V.off, V.Adia.get(), n, k, P, AP, fin);
        else launch_csr_block_dot(V.A.rowptr, V.A.cols, V.A.vals, n, k, P, AP, bs.l32[0].sA, fin);
        return;
    }
    if (H.is_finest(A) && H.opts.precision == RB_PREC_FP64 && H.lv64[0].dia) {
        const Level<double>& V = H.lv64[0];
        launch_dia_block_dot(V.off, V.Adia.get(), n, k, P, AP, fin);
        return;
    }
    launch_csr_block_dot(A.rowptr.get(), A.cols.get(), A.vals.get(), n, k, P, AP, bs.sA0, fin);
}

void block_residual64(BlockState& bs, const rb_csr_s& A, const double* X, const double* B,
                      double* R) {
    launch_csr_block(A.rowptr.get(), A.cols.get(), A.vals.get(), (long)A.n_rows, bs.k, X,
                     BResidual<double, double>{B, R}, bs.sA0);
}

}  // namespace

BlockState& Hierarchy::block_state(int k) {
    RB_REQUIRE(k >= 2 && k <= kMaxBlockK, "block: k must be in 2..32");
    if (blk && blk->k == k) return *blk;
    release_graphs();
    blk.reset();
    auto s = std::make_shared<BlockState>();
    s->k = k;
    const long n = master[0].A->n_rows;
    const size_t m = (size_t)std::max<long>(n, 1) * k;
    s->R.alloc(m);
    s->Z.alloc(m);
    s->P.alloc(m);
    s->AP.alloc(m);
    s->Rt.alloc(m);
    s->scal.alloc(1);
    RB_CUDA(cudaMallocHost(&s->host, sizeof(BlockScal)));
    if (opts.precision == RB_PREC_FP32) build_block_levels(lv32, s->l32, k);
    else build_block_levels(lv64, s->l64, k);
    s->sA0 = tune_split(view(*master[0].A), k, s->P.get(), s->AP.get(), "bA0");
    blk = s;
    return *blk;
}

// Z = M B for k columns (one block V-cycle from a zero guess).
void Hierarchy::cycle_block(double* Z, const double* B, int k) {
    BlockState& bs = block_state(k);
    run_graph(bkey("cycB", k, Z, B, nullptr), [&] { block_cycle64(*this, bs, Z, B); });
}

int Hierarchy::pcg_block(const rb_csr_s& A, double* X, const double* B, int k, double tol,
                         int max_iter, int* iters, double* relres) {
    const long n = A.n_rows;
    RB_REQUIRE(n == master[0].A->n_rows, "block PCG: A and the hierarchy differ in size");
    RB_REQUIRE(k >= 2 && k <= kMaxBlockK, "block PCG: k must be in 2..32");
    RB_REQUIRE(opts.relax_type == RB_RELAX_JACOBI || opts.relax_type == RB_RELAX_L1JACOBI,
               "block PCG: the smoother must be Jacobi or L1-Jacobi");
    if (max_iter <= 0) max_iter = (int)(1.3 * n) + 2;
    BlockState& bs = block_state(k);
    BlockScal* S = bs.scal.get();
    BlockScal& h = *bs.host;
    double* R = bs.R.get();
    double* Z = bs.Z.get();
    double* P = bs.P.get();
    double* AP = bs.AP.get();
    auto read = [&]() {
        RB_CUDA(cudaMemcpyAsync(&h, S, sizeof(BlockScal), cudaMemcpyDeviceToHost, stream()));
        RB_CUDA(cudaStreamSynchronize(stream()));
    };
    auto push_active = [&]() {
        RB_CUDA(cudaMemcpyAsync(S->active, h.active, sizeof(int) * kMaxBlockK,
                                cudaMemcpyHostToDevice, stream()));
    };
    RB_CUDA(cudaMemsetAsync(S, 0, sizeof(BlockScal), stream()));
    // ||b_c||
    launch_block_dot(n, k, B, B, FinBTmp{S});
    read();
    std::vector<double> bnorm(k);
    for (int c = 0; c < k; c++) {
        bnorm[c] = std::sqrt(h.tmp[c]);
        h.active[c] = bnorm[c] > 0.0 ? 1 : 0;
        iters[c] = 0;
        relres[c] = 0.0;
    }
    push_active();
    // In the FP32 form the block cycle reads R in FP32 (written by the update
    // kernel, or converted after a full residual) and its FP32 output z is
    // read directly by the r.z dots and the P update, without an FP64 copy.
    const bool f32 = opts.precision == RB_PREC_FP32;
    const long nk = n * k;
    const int KP = pow2_at_least(k);
    float* r32 = f32 ? bs.l32[0].b.get() : nullptr;
    const float* z32 = f32 ? bs.l32[0].x.get() : nullptr;
    auto to_r32 = [&]() {
        k_convert<float, double><<<grid_for(nk, 256), 256, 0, stream()>>>(nk, R, r32);
        RB_CHECK_LAUNCH();
    };
    auto precond = [&]() {   // z = M r from a zero guess
        if (f32) block_cycle_level(*this, lv32, bs.l32, 0, bs.l32[0].x.get(), r32, true, k);
        else block_cycle_level(*this, lv64, bs.l64, 0, Z, R, true, k);
    };
    auto dot_rz = [&](auto fin) {
        if (f32) launch_block_dot(n, k, R, z32, fin);
        else launch_block_dot(n, k, R, (const double*)Z, fin);
    };
    auto p_update = [&](int restart) {
        const unsigned g = grid_for(n * KP, 256);
        RB_BLOCK_KP_SWITCH(KP, {
            if (f32) k_bcg_p<kKP, float><<<g, 256, 0, stream()>>>(n, k, P, z32, S, restart);
            else k_bcg_p<kKP, double><<<g, 256, 0, stream()>>>(n, k, P, Z, S, restart);
        });
        RB_CHECK_LAUNCH();
    };
    // R = B - A X ; Z = M R ; P = Z ; rz, rr
    auto restart = [&]() {
        block_residual64(bs, A, X, B, R);
        if (f32) to_r32();
        precond();
        p_update(1);
        dot_rz(FinBSetRZ{S});
        launch_block_dot(n, k, R, R, FinBRR{S});
    };
    restart();
    read();
    // per-column stop: the recursive residual meets tol, then the true one
    // (B - A X) confirms; returns true when every column has stopped
    int iter = 0;
    auto check = [&]() -> bool {
        bool candidate = false;
        for (int c = 0; c < k; c++)
            if (h.active[c] && std::sqrt(h.rr[c]) <= tol * bnorm[c]) candidate = true;
        if (candidate) {
            block_residual64(bs, A, X, B, bs.Rt.get());
            launch_block_dot(n, k, bs.Rt.get(), bs.Rt.get(), FinBTmp{S});
            read();
            bool failed = false;
            for (int c = 0; c < k; c++) {
                if (!h.active[c]) continue;
                const double tr = std::sqrt(h.tmp[c]);
                if (std::sqrt(h.rr[c]) <= tol * bnorm[c]) {
                    if (tr <= tol * bnorm[c]) {
                        h.active[c] = 0;
                        iters[c] = iter;
                        relres[c] = tr / bnorm[c];
                    } else {
                        failed = true;
                    }
                }
            }
            push_active();
            if (failed) {
                // the recurrence drifted from the true residual: restart it
                restart();
                read();
            }
        }
        for (int c = 0; c < k; c++)
            if (h.active[c]) return false;
        return true;
    };
    if (check()) return RB_OK;
    auto body = [&](bool full_r) {
        block_outer_apply(*this, bs, A, P, AP);
        const unsigned g = block_grid(n, KP, 1);
        ReduceSlot rs = global_reduce_slot((int)g * kMaxBlockK);
        float* r32_out = (f32 && !full_r) ? r32 : nullptr;
        RB_BLOCK_KP_SWITCH(KP, {
            k_bcg_update<kKP><<<g, 256, 0, stream()>>>(n, k, X, R, P, AP, S, rs, FinBRR{S}, r32_out);
        });
        RB_CHECK_LAUNCH();
        if (full_r) {
            block_residual64(bs, A, X, B, R);
            launch_block_dot(n, k, R, R, FinBRR{S});
            if (f32) to_r32();
        }
        precond();
        dot_rz(FinBRZ{S});
    };
    int status = RB_ERR_NOT_CONVERGED;
    while (iter < max_iter) {
        iter++;
        const bool full_r = iter % 10 == 0;
        run_graph(bkey(full_r ? "pcgBF" : "pcgB", k, X, B, &A), [&] { body(full_r); });
        read();
        if (h.breakdown) return RB_ERR_BREAKDOWN;
        if (check()) { status = RB_OK; break; }
        p_update(0);
    }
    if (status != RB_OK) {
        for (int c = 0; c < k; c++)
            if (h.active[c]) {
                iters[c] = iter;
                relres[c] = std::sqrt(h.rr[c]) / bnorm[c];
            }
    }
    last_iters = iter;
    return status;
}

}  // namespace rb
