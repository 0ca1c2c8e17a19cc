// hierarchy.cuh -- the device AMG hierarchy (ParMultilevel at world size 1).
#pragma once

#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "blas1.cuh"
#include "dia.cuh"
#include "rb_internal.cuh"
#include "tail_cycle.cuh"
#include "tiled.cuh"

namespace rb {

// Autotuner decisions keyed by operator, size and value width (persisted
// when RAPTOR_B200_TUNE_CACHE names a file).
struct TuneCache {
    std::map<std::string, int> m;
    bool loaded = false;
    std::string path;
};
TuneCache& tune_cache();
void tune_save();
std::string tune_key(const char* op, long n, long long nnz, int vbytes);

// The autotuner times each candidate cold, as the cycle runs it: before every
// timed launch a buffer larger than the L2 is overwritten, and then `warm`
// (the vector the product gathers from, just written by the previous step of
// a cycle) is read back into the L2, so the operator's values and indices
// stream from HBM while its input vector is cached.  Back-to-back repeats
// instead keep part of a matrix below the L2's size resident and favour
// schedules that do not win inside a cycle.
void tune_cold_l2(const void* warm, size_t bytes);
constexpr int kTuneReps = 5;

// Milliseconds of the fastest of kTuneReps cold launches of fn (after one
// untimed launch that takes any first-launch costs).
template <class F>
float time_launch(F&& fn, const void* warm = nullptr, size_t warm_bytes = 0) {
    cudaEvent_t e0, e1;
    RB_CUDA(cudaEventCreate(&e0));
    RB_CUDA(cudaEventCreate(&e1));
    fn();
    float best = 1e30f;
    for (int rep = 0; rep < kTuneReps; rep++) {
        tune_cold_l2(warm, warm_bytes);
        RB_CUDA(cudaEventRecord(e0, stream()));
        fn();
        RB_CUDA(cudaEventRecord(e1, stream()));
        RB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        RB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = ms < best ? ms : best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

struct BlockState;   // k right-hand-side buffers and tile shapes (block.cu)

// FP64 result of setup for one level (multilevel/par_level.hpp:15-43).
struct MasterLevel {
    std::unique_ptr<rb_csr_s> A;   // diagonal first
    std::unique_ptr<rb_csr_s> P;   // n_l x n_{l+1}
    std::unique_ptr<rb_csr_s> R;   // P^T, stored so restriction is a gather
    DevArray<int> states;          // C/F splitting
};

// Cycle data of one level in the cycle precision T.
// 16-bit column offsets of a CSR operator whose rows each span fewer than
// 65536 columns (column = base[row] + c16[j]); used when the autotuner
// finds it faster than the 32-bit indices.
// The same record holds the chunk windows of the shared-memory schedule
// (tiled.cuh) when it is built for the operator.
struct Idx16 {
    bool on = false;
    DevArray<int> base;
    DevArray<unsigned short> c16;
    int tchunks = 0, trows = 0, twmax = 0;   // tiles: chunks, rows a chunk, largest window
    DevArray<int> tlo, thi;
};

// rows of M times x with the epilogue, through 16- or 32-bit column indices,
// on the strided, blocked (kRowsBlocked) or shared-memory (kRowsTiled)
// schedule the lanes value G names
template <typename T, typename TX, class Epi>
void rows_op(const CsrView<T>& M, const Idx16& I, long n_rows, const TX* x, Epi epi, int G) {
    if constexpr (HasRowSkip<Epi>::value) {
        G &= kRowsBlocked - 1;   // row-gated epilogues run the strided schedule
    } else if ((G & kRowsTiled) && I.tchunks) {
        const int g = G & (kRowsBlocked - 1);
        if (I.on)
            launch_tiled<T, TX, Epi, true>(n_rows, M.rowptr, M.cols, I.base.get(), I.c16.get(),
                                           M.vals, x, I.tlo.get(), I.thi.get(), I.trows,
                                           I.tchunks, I.twmax, epi, g);
        else
            launch_tiled<T, TX, Epi, false>(n_rows, M.rowptr, M.cols, nullptr, nullptr, M.vals, x,
                                            I.tlo.get(), I.thi.get(), I.trows, I.tchunks,
                                            I.twmax, epi, g);
        return;
    }
    G &= ~kRowsTiled;
    if (I.on) launch_rows16(M.rowptr, I.base.get(), I.c16.get(), M.vals, n_rows, M.nnz, x, epi, G);
    else launch_rows(M.rowptr, M.cols, M.vals, n_rows, M.nnz, x, epi, G);
}

template <typename T>
struct Level {
    int n = 0;
    CsrView<T> A, P, R;
    Idx16 A16, P16, R16;
    DevArray<T> Avals, Pvals, Rvals;   // value copies when T != double
    DevArray<T> dinv;                  // w / a_ii (Jacobi) or w / sum|a_ij| (L1)
    DevArray<int> colour_rows;         // rows grouped by colour (multicolour SOR)
    std::vector<int> colour_ptr;
    DevArray<T> x, b, r, xt;
    int gA = 0, gP = 0, gR = 0;        // lanes per row picked by the autotuner
    bool dia = false;                  // A_l by diagonals (the autotuner's pick)
    bool fuse_first = false;           // first sweep fused with the residual (timed pick)
    DiaOff off{};
    DevArray<T> Adia;
    DevArray<unsigned> dmask;          // constant-coefficient form (DiaOff::mask)
    void alloc_vectors();

    // y-epilogue over the rows of A_l times x, in whichever format was picked
    template <typename TX, class Epi>
    void apply_A(const TX* xin, Epi epi) const {
        if constexpr (HasRowSkip<Epi>::value) rows_op(A, A16, n, xin, epi, gA);
        else if (dia) launch_dia(off, Adia.get(), n, xin, epi);
        else rows_op(A, A16, n, xin, epi, gA);
    }
};

struct Hierarchy {
    rb_amg_opts opts{};
    std::vector<MasterLevel> master;
    std::vector<Level<double>> lv64;
    std::vector<Level<float>> lv32;
    int coarse_n = 0;
    DevArray<double> lu;
    DevArray<double> cinv;   // inverse of the coarse matrix (coarse_n <= kCoarseInvMax)
    DevArray<int> piv;
    // Krylov work vectors (finest size) and device scalars
    DevArray<double> kr, kz, kp, kAp, ks, kAs, krs, kph, ksh;
    DevArray<KScal> scal;
    KScal* host_scal = nullptr;
    PcgCtl* host_ctl = nullptr;   // pinned staging of the device-side loop state
    int gA0 = 0;
    bool use_graphs = true;
    // the levels of an uneven batch: every operator on the strided schedule
    // in CSR (16- or 32-bit indices), which the row gates of stopped systems
    // apply to
    bool strided_only = false;
    // bottom of the cycle (levels tail_from .. L-1) in one launch of one
    // cluster of tail_ctas CTAs (tail_cycle.cuh); tail_from = -1: off
    int tail_from = -1;
    int tail_ctas = 0;
    DevArray<LevelDesc<double>> tdesc64;
    DevArray<LevelDesc<float>> tdesc32;
    template <typename T>
    void build_tail(std::vector<Level<T>>& lv, DevArray<LevelDesc<T>>& desc, int from);
    template <typename T>
    void launch_tail(std::vector<Level<T>>& lv, DevArray<LevelDesc<T>>& desc);
    template <typename T>
    void tune_tail(std::vector<Level<T>>& lv, DevArray<LevelDesc<T>>& desc);
    std::vector<double> tail_ms;   // cycle ms per candidate start (tuning record)
    std::map<std::string, cudaGraphExec_t> graphs;
    std::map<std::string, long long> graph_kernels;
    // the matrix handed to setup: PCG on it reads the hierarchy's copies of
    // A_0 (the same values, stored by diagonals / in the cycle precision)
    const rb_csr_s* src_A = nullptr;
    bool is_finest(const rb_csr_s& A) const {
        return &A == master[0].A.get() ||
               (&A == src_A && A.nnz == master[0].A->nnz && A.n_rows == master[0].A->n_rows);
    }
    // every value of A_0 is exactly representable in FP32: the FP32 copy of
    // A_0 (FP64 accumulation) then is the operator itself, and residuals of
    // the outer iteration read it instead of the FP64 CSR matrix
    bool a0_fp32_exact = false;
    // A_0 by diagonals in FP64 for the outer operator of the FP32 form when
    // A_0's values are not exact in FP32 (then the FP32 copy is a perturbed
    // operator, which an ill-conditioned problem does not tolerate)
    Level<double> a0_64;
    void true_residual(const rb_csr_s& A, const double* x, const double* b, double* r);
    double setup_seconds = 0;
    int last_iters = 0;

    ~Hierarchy();
    // cycle_data = false builds the FP64 levels only (a member of a batch)
    void setup(const rb_csr_s& A, const rb_amg_opts& o, const double* weights_host,
               bool cycle_data = true);
    void build_cycle_data();
    template <typename T>
    void build_levels(std::vector<Level<T>>& lv);
    int num_levels() const { return (int)master.size(); }

    template <typename T>
    void smooth(Level<T>& V, T*& cur, T*& other, const T* b, bool x_zero);
    template <typename T>
    void cycle_level(std::vector<Level<T>>& lv, int l, T* x, const T* b, bool x_zero);
    void cycle64(double* x, const double* b, bool x_zero);
    void cycle(double* x, const double* b, bool x_zero);
    void run_graph(const std::string& key, const std::function<void()>& fn);
    void run_while_graph(const std::string& key,
                         const std::function<void(cudaGraphConditionalHandle)>& fn);
    void release_graphs();

    void dot_into(const double* a, const double* b, long n, double* field);
    double norm64(const double* v, long n);
    KScal read_scal();

    // profiling (multilevel/par_multilevel.hpp:343-456 keeps per-level
    // solve_times; here CUDA events bracket each operation of one cycle)
    std::vector<std::pair<int, cudaEvent_t>>* prof = nullptr;
    void mark(int slot);
    std::vector<double> profile_cycle();
    double time_operator(int level, int op, int reps);

    int solve(double* x, const double* b, double* hist, int cap, int* iters);
    // outer A p fused with p.Ap on the finest level: from the FP64 operator,
    // or from the cycle-precision copy of A_0 with FP64 accumulation
    template <class Fin>
    void outer_apply(const rb_csr_s& A, bool lowprec, const double* p, double* Ap, Fin fin);
    int pcg(const rb_csr_s& A, double* x, const double* b, double tol, int max_iter, int mode,
            double* hist, int cap, int* n_hist);
    size_t device_bytes() const;

    // k right-hand sides at once (block.cu): X and B are n x k blocks, entry
    // (i, c) at i * k + c; per-column CG scalars, one shared hierarchy.
    // adjoint solves (adjoint.cu): symmetry of the last operator checked, and
    // for a nonsymmetric one the hierarchy of the transposed cycle
    const rb_csr_s* adj_A = nullptr;
    bool adj_sym = false;
    std::unique_ptr<Hierarchy> adj;
    std::unique_ptr<rb_csr_s> adj_AT;

    std::shared_ptr<BlockState> blk;
    BlockState& block_state(int k);
    void cycle_block(double* Z, const double* B, int k);
    int pcg_block(const rb_csr_s& A, double* X, const double* B, int k, double tol, int max_iter,
                  int* iters, double* relres);
};

int krylov_cg(const rb_csr_s& A, double* x, const double* b, double tol, int max_iter,
              double* hist, int cap, int* n_hist);
int krylov_bicgstab(const rb_csr_s& A, Hierarchy* ml, double* x, const double* b, double tol,
                    int max_iter, double* hist, int cap, int* n_hist);
// A^T lambda = g through the hierarchy built for A (adjoint.cu)
int adjoint_solve(const rb_csr_s& A, Hierarchy& H, double* lambda, const double* g, double tol,
                  int max_iter, int* iters, double* relres);

}  // namespace rb

struct rb_amg_s {
    rb::Hierarchy h;
};
