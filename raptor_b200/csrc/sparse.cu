// sparse.cu -- CSR containers, row canonicalisation, transpose, scans,
// deterministic reductions and the FP64 SpMV primitives of the C ABI.
#include <cub/cub.cuh>

#include <climits>
#include <mutex>
#include <unordered_map>

#include "rb_internal.cuh"
#include "spmv.cuh"

namespace rb {

// ------------------------------------------------------------- context --
namespace {
cudaStream_t g_stream = nullptr;
cudaStream_t g_own_stream = nullptr;
int g_sms = 0;
thread_local std::string g_last_error;
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }

long long& launch_counter() {
    static long long c = 0;
    return c;
}
long long& device_alloc_counter() {
    static long long c = 0;
    return c;
}
const char* last_error_cstr() { return g_last_error.c_str(); }

cudaStream_t stream() {
    if (!g_stream) {
        if (!g_own_stream) RB_CUDA(cudaStreamCreateWithFlags(&g_own_stream, cudaStreamNonBlocking));
        g_stream = g_own_stream;
    }
    return g_stream;
}

void set_stream(cudaStream_t s) { g_stream = s ? s : nullptr; }

int sm_count() {
    if (!g_sms) {
        int dev = 0;
        RB_CUDA(cudaGetDevice(&dev));
        RB_CUDA(cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    return g_sms;
}

void tune_cold_l2(const void* warm, size_t bytes) {
    // 192 MB, above the 126 MB L2; allocated once and kept for the process
    constexpr size_t kFlush = (size_t)192 << 20;
    static DevArray<char>* buf = nullptr;
    if (!buf) {
        buf = new DevArray<char>();
        buf->alloc(kFlush);
    }
    RB_CUDA(cudaMemsetAsync(buf->get(), 0, kFlush, stream()));
    if (warm && bytes)
        RB_CUDA(cudaMemcpyAsync(buf->get(), warm, bytes < kFlush ? bytes : kFlush,
                                cudaMemcpyDeviceToDevice, stream()));
}

int resident_blocks_per_sm(const void* fn, int threads) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(fn);
    if (it != cache.end()) return it->second;
    int b = 0;
    RB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, threads, 0));
    if (b < 1) b = 1;
    cache[fn] = b;
    return b;
}

int grid_per_sm(const char* env, int dflt) {
    const char* v = getenv(env);
    const int k = v ? atoi(v) : 0;
    return k > 0 ? k : dflt;
}

rb_csr_s* new_csr(int n_rows, int n_cols, long long nnz) {
    RB_REQUIRE(n_rows >= 0 && n_cols >= 0 && nnz >= 0, "negative matrix dimension");
    RB_REQUIRE(nnz <= INT_MAX, "matrix has more than 2^31-1 nonzeros (int32 indices)");
    auto* A = new rb_csr_s();
    A->n_rows = n_rows;
    A->n_cols = n_cols;
    A->nnz = nnz;
    A->rowptr.alloc((size_t)n_rows + 1);
    A->cols.alloc((size_t)(nnz > 0 ? nnz : 1));
    A->vals.alloc((size_t)(nnz > 0 ? nnz : 1));
    return A;
}

// ------------------------------------------------------------------ scan --
__global__ void k_scan_tail(const int* in, int* out, int n, long long* total) {
    long long t = (n > 0) ? (long long)out[n - 1] + (long long)in[n - 1] : 0;
    *total = t;
    out[n] = (int)t;
}

long long exclusive_scan(const int* in, int* out, int n) {
    if (n == 0) {
        RB_CUDA(cudaMemsetAsync(out, 0, sizeof(int), stream()));
        return 0;
    }
    size_t bytes = 0;
    RB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, stream()));
    DevArray<char> tmp(bytes + 16);
    RB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, in, out, n, stream()));
    DevArray<long long> tot(1);
    k_scan_tail<<<1, 1, 0, stream()>>>(in, out, n, tot.get());
    RB_CHECK_LAUNCH();
    long long t = read_scalar(tot.get());
    RB_REQUIRE(t >= 0 && t <= INT_MAX, "prefix sum exceeds the int32 index range");
    return t;
}

// -------------------------------------------------- row canonicalisation --
// Insertion sort of each row by column (CSRMatrix::sort, core/matrix.cpp
// :588-618), then the diagonal moved to the front (move_diag_helper,
// :730-786).  One thread per row: rows of the path are short.
__global__ void k_sort_rows(int n, const int* __restrict__ rp, int* cols, double* vals,
                            int diag_first) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int s = rp[i], e = rp[i + 1];
    for (int j = s + 1; j < e; j++) {
        int c = cols[j];
        double v = vals[j];
        int k = j - 1;
        while (k >= s && cols[k] > c) {
            cols[k + 1] = cols[k];
            vals[k + 1] = vals[k];
            k--;
        }
        cols[k + 1] = c;
        vals[k + 1] = v;
    }
    if (diag_first) {
        for (int j = s; j < e; j++) {
            if (cols[j] == i) {
                double t = vals[j];
                for (int k = j; k > s; k--) {
                    cols[k] = cols[k - 1];
                    vals[k] = vals[k - 1];
                }
                cols[s] = i;
                vals[s] = t;
                break;
            }
        }
    }
}

void sort_rows_diag_first(rb_csr_s& A, bool diag_first) {
    if (A.n_rows == 0) return;
    k_sort_rows<<<grid_for(A.n_rows, 256), 256, 0, stream()>>>(A.n_rows, A.rowptr.get(),
                                                                 A.cols.get(), A.vals.get(),
                                                                 diag_first ? 1 : 0);
    RB_CHECK_LAUNCH();
}

// Deep copy on the device.
rb_csr_s* clone_csr(const rb_csr_s& M) {
    rb_csr_s* C = new_csr(M.n_rows, M.n_cols, M.nnz);
    RB_CUDA(cudaMemcpyAsync(C->rowptr.get(), M.rowptr.get(), sizeof(int) * ((size_t)M.n_rows + 1),
                            cudaMemcpyDeviceToDevice, stream()));
    if (M.nnz) {
        RB_CUDA(cudaMemcpyAsync(C->cols.get(), M.cols.get(), sizeof(int) * M.nnz,
                                cudaMemcpyDeviceToDevice, stream()));
        RB_CUDA(cudaMemcpyAsync(C->vals.get(), M.vals.get(), sizeof(double) * M.nnz,
                                cudaMemcpyDeviceToDevice, stream()));
    }
    return C;
}

// ------------------------------------------------------------ transpose --
__global__ void k_count_cols(long long nnz, const int* __restrict__ cols, int* cnt) {
    long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < nnz) atomicAdd(cnt + cols[j], 1);
}

__global__ void k_scatter_T(int n, const int* __restrict__ rp, const int* __restrict__ cols,
                            const double* __restrict__ vals, int* fill, int* tcols,
                            double* tvals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int j = rp[i]; j < rp[i + 1]; j++) {
        int c = cols[j];
        int p = atomicAdd(fill + c, 1);
        tcols[p] = i;
        tvals[p] = vals[j];
    }
}

rb_csr_s* transpose(const rb_csr_s& A) {
    rb_csr_s* T = new_csr(A.n_cols, A.n_rows, A.nnz);
    DevArray<int> cnt((size_t)A.n_cols + 1);
    cnt.zero();
    if (A.nnz)
        k_count_cols<<<grid_for(A.nnz, 256), 256, 0, stream()>>>(A.nnz, A.cols.get(), cnt.get());
    RB_CHECK_LAUNCH();
    exclusive_scan(cnt.get(), T->rowptr.get(), A.n_cols);
    RB_CUDA(cudaMemcpyAsync(cnt.get(), T->rowptr.get(), sizeof(int) * A.n_cols,
                            cudaMemcpyDeviceToDevice, stream()));
    if (A.n_rows)
        k_scatter_T<<<grid_for(A.n_rows, 256), 256, 0, stream()>>>(
            A.n_rows, A.rowptr.get(), A.cols.get(), A.vals.get(), cnt.get(), T->cols.get(),
            T->vals.get());
    RB_CHECK_LAUNCH();
    // atomics leave each row in arbitrary order: sort by source row
    sort_rows_diag_first(*T, false);
    return T;
}

// ------------------------------------------------- transposed product --
__global__ void k_iota_vals(long long nnz, double* v) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x)
        v[k] = (double)k;
}

__global__ void k_to_int(long long nnz, const double* v, int* out) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x)
        out[k] = (int)v[k];
}

// y_j = sum over the entries of row j of A^T of vals[src] * x[row]: 8 lanes
// per row, each lane a fixed stride of the row, then a fixed shuffle tree,
// so the result does not depend on scheduling.
__global__ void __launch_bounds__(256)
k_spmv_T_map(int n, const int* __restrict__ rp, const int* __restrict__ rows,
             const int* __restrict__ src, const double* __restrict__ vals,
             const double* __restrict__ x, double* __restrict__ y) {
    constexpr int G = 8;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long j = t / G;
    const int g = threadIdx.x & (G - 1);
    double s = 0.0;
    if (j < n)
        for (int k = rp[j] + g; k < rp[j + 1]; k += G) s += vals[src[k]] * x[rows[k]];
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, G);
    if (j < n && g == 0) y[j] = s;
}

void spmv_T64(rb_csr_s& A, const double* x, double* y) {
    if (!A.tmap) {
        // transpose a copy of A whose values are the entry positions: the
        // transposed values are then the source positions, in the order the
        // deterministic transpose leaves its rows
        std::unique_ptr<rb_csr_s> I(clone_csr(A));
        if (A.nnz)
            k_iota_vals<<<grid_for(A.nnz, 256), 256, 0, stream()>>>(A.nnz, I->vals.get());
        RB_CHECK_LAUNCH();
        std::unique_ptr<rb_csr_s> T(transpose(*I));
        auto m = std::make_unique<TransposeMap>();
        m->src.alloc((size_t)A.nnz + 1);
        if (A.nnz)
            k_to_int<<<grid_for(A.nnz, 256), 256, 0, stream()>>>(A.nnz, T->vals.get(),
                                                                  m->src.get());
        RB_CHECK_LAUNCH();
        m->rowptr = std::move(T->rowptr);
        m->rows = std::move(T->cols);
        A.tmap = std::move(m);
    }
    if (A.n_cols)
        k_spmv_T_map<<<grid_for((long)A.n_cols * 8, 256), 256, 0, stream()>>>(
            A.n_cols, A.tmap->rowptr.get(), A.tmap->rows.get(), A.tmap->src.get(), A.vals.get(),
            x, y);
    RB_CHECK_LAUNCH();
}

// ---------------------------------------------------------------- dots --
struct FinStore {
    double* out;
    __device__ void operator()(double t) const { *out = t; }
};

__global__ void __launch_bounds__(256) k_dot(const double* __restrict__ a,
                                             const double* __restrict__ b, long n,
                                             ReduceSlot rs, FinStore fin) {
    double t = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        t += a[i] * b[i];
    block_reduce_finish(t, rs, fin);
}

namespace {
struct ReduceScratch {
    DevArray<double> partials;
    DevArray<unsigned> ticket;
    std::once_flag once;
};
ReduceScratch& scratch() {
    static ReduceScratch s;
    return s;
}
}  // namespace

// One scratch for every reduction on the library stream.  It is allocated
// once and never moved, because CUDA graphs capture its address.
constexpr int kMaxReduceGrid = 1 << 16;

ReduceSlot global_reduce_slot(int grid) {
    auto& s = scratch();
    RB_REQUIRE(grid <= kMaxReduceGrid, "reduction grid too large");
    if (!s.partials.size()) {
        s.partials.alloc(kMaxReduceGrid);
        s.ticket.alloc(1);
        s.ticket.zero();
        RB_CUDA(cudaStreamSynchronize(stream()));
    }
    return ReduceSlot{s.partials.get(), s.ticket.get()};
}

void dot_async(const double* a, const double* b, int n, double* result_dev) {
    const int grid = std::max(1, std::min(sm_count() * 4, (int)((n + 255) / 256)));
    ReduceSlot rs = global_reduce_slot(grid);
    k_dot<<<grid, 256, 0, stream()>>>(a, b, n, rs, FinStore{result_dev});
    RB_CHECK_LAUNCH();
}

// ------------------------------------------------------- FP64 SpMV ops --
void spmv64(const CsrView<double>& A, const double* x, double* y, int lanes) {
    launch_rows(A.rowptr, A.cols, A.vals, A.n_rows, A.nnz, x, EpiStore<double>{y}, lanes);
}

void residual64(const CsrView<double>& A, const double* x, const double* b, double* r,
                int lanes) {
    launch_rows(A.rowptr, A.cols, A.vals, A.n_rows, A.nnz, x, EpiResidual<double, double>{b, r},
                lanes);
}

void spmv_append64(const CsrView<double>& A, const double* x, double* y, int lanes) {
    launch_rows(A.rowptr, A.cols, A.vals, A.n_rows, A.nnz, x, EpiAppend<double>{y}, lanes);
}

int handle_lanes(rb_csr_s& A, const double* x) {
    if (A.lanes) return A.lanes;
    if (A.n_rows < 4096 || A.nnz == 0) return A.lanes = pick_group(A.n_rows, A.nnz);
    // products into a scratch vector of its own (the caller's output may be
    // an input too, as in mult_append), each schedule timed over 3 launches
    DevArray<double> y((size_t)A.n_rows);
    static const int cands[10] = {2, 4, 8, 16, 32, kRowsBlocked | 4, kRowsBlocked | 8,
                                  kRowsBlocked | 16, kRowsBlocked | 32, 1};
    cudaEvent_t e0, e1;
    RB_CUDA(cudaEventCreate(&e0));
    RB_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int bestG = pick_group(A.n_rows, A.nnz);
    const CsrView<double> v = view(A);
    for (int G : cands) {
        spmv64(v, x, y.get(), G);
        RB_CUDA(cudaEventRecord(e0, stream()));
        for (int rep = 0; rep < 3; rep++) spmv64(v, x, y.get(), G);
        RB_CUDA(cudaEventRecord(e1, stream()));
        RB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        RB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) { best = ms; bestG = G; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return A.lanes = bestG;
}

}  // namespace rb
