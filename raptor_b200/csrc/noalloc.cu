// noalloc.cu -- ||b - A x||_2 without any device allocation.
//
// Every other entry point of this library may allocate device memory
// (cudaMalloc) for its temporaries.  Some callers cannot allow that:
// runtimes that hand the library a fixed memory budget and forbid any
// allocation once a solve is under way (an allocation there can fail), and
// real-time loops in which cudaMalloc's implicit device synchronisation would
// break the deadline.  rb_residual_norm_noalloc serves them:
// it computes the quantity ParMultilevel::solve checks after every cycle,
// the 2-norm of the residual b - A x, in one kernel whose only temporary
// storage -- the per-block partial sums of the deterministic two-stage
// reduction and the block-completion counter -- lives in the file-scope
// device array below.
//
// Limits and sharing:
//   * at most kNoAllocMaxRows = 16777216 rows: each block reduces a fixed
//     run of kRowsPerBlock rows and the array holds one partial per block;
//   * the array exists once per device that loads this library and is held
//     until the process exits (128 KiB + 256 bytes);
//   * every call shares it and it keeps the last call's contents: the
//     completion counter is cleared at the start of each call, the partials
//     are always written before they are read.  Calls that overlap on the
//     GPU (two streams, or two host threads, at once) race on it;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (in host code the name is only a host-side
//     stand-in), with that device current; make that first call before any
//     stream capture begins.
// Error messages stay within the short-string buffer of the library's error
// string, so even a rejected call allocates nothing.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/raptor_b200.h"

namespace rb {
void set_last_error(const std::string& msg);
long long& launch_counter();
}

namespace {

constexpr int kRowsPerBlock = 1024;
constexpr int kNoAllocMaxBlocks = 16384;
constexpr long long kNoAllocMaxRows = (long long)kRowsPerBlock * kNoAllocMaxBlocks;
constexpr int kBlock = 256;
constexpr int kLanes = 8;   // lanes per row

// partials[kNoAllocMaxBlocks] doubles, then the completion counter
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocMaxBlocks * sizeof(double) + 256];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

__global__ void __launch_bounds__(kBlock)
k_residual_norm(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                const double* __restrict__ cv, const double* __restrict__ x,
                const double* __restrict__ b, double* out, unsigned char* scratch) {
    double* partials = reinterpret_cast<double*>(scratch);
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kNoAllocMaxBlocks * sizeof(double));
    const int lane = threadIdx.x & 31, sub = lane / kLanes, gl = lane & (kLanes - 1);
    const int warp = threadIdx.x >> 5;
    const int rows_per_pass = (kBlock / 32) * (32 / kLanes);
    const long first = (long)blockIdx.x * kRowsPerBlock;
    double acc = 0.0;
    for (int base = 0; base < kRowsPerBlock; base += rows_per_pass) {
        const long row = first + base + warp * (32 / kLanes) + sub;
        const bool valid = row < n;
        double s = 0.0;
        if (valid)
            for (int j = rp[row] + gl; j < rp[row + 1]; j += kLanes) s += cv[j] * x[ci[j]];
#pragma unroll
        for (int o = kLanes / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, kLanes);
        if (valid && gl == 0) {
            const double r = b[row] - s;
            acc += r * r;
        }
    }
    // block tree, then the last block to finish sums the partials in order
    __shared__ double wsum[kBlock / 32];
    __shared__ bool last;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) wsum[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; w++) t += wsum[w];
        partials[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += kBlock) t += ((volatile double*)partials)[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    __syncthreads();
    if (lane == 0) wsum[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < kBlock / 32; w++) tot += wsum[w];
        *out = sqrt(tot);
        *ticket = 0u;
    }
}

int fail(int code, const char* msg) {
    rb::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" int rb_residual_norm_noalloc(int n_rows, const int* rowptr, const int* cols,
                                        const double* vals, const double* x, const double* b,
                                        double* norm_out, void* stream) {
    rb::set_last_error("");
    if (n_rows < 0) return fail(RB_ERR_INVALID, "n_rows < 0");
    if ((long long)n_rows > kNoAllocMaxRows) return fail(RB_ERR_INVALID, "n_rows > 2^24");
    if (!rowptr || !norm_out || (n_rows > 0 && (!cols || !vals || !x || !b)))
        return fail(RB_ERR_INVALID, "NULL argument");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(RB_ERR_NO_DEVICE, "no CUDA device");
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> g(g_scratch_mutex);
        if (!g_scratch_addr[dev]) {
            // first call on this device (it is current): resolve the array's
            // device address; this must precede any stream capture
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
                return fail(RB_ERR_CUDA, "symbol lookup");
            g_scratch_addr[dev] = p;
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    // an error left pending by earlier, unrelated work is not this call's
    (void)cudaGetLastError();
    const int blocks = n_rows > 0 ? (int)((n_rows + kRowsPerBlock - 1) / kRowsPerBlock) : 1;
    // the completion counter must start at zero
    if (cudaMemsetAsync((unsigned char*)scratch + kNoAllocMaxBlocks * sizeof(double), 0,
                        sizeof(unsigned), st) != cudaSuccess)
        return fail(RB_ERR_CUDA, "counter clear");
    k_residual_norm<<<blocks, kBlock, 0, st>>>(n_rows, rowptr, cols, vals, x, b, norm_out,
                                               (unsigned char*)scratch);
    if (cudaGetLastError() != cudaSuccess) return fail(RB_ERR_CUDA, "kernel launch");
    ++rb::launch_counter();
    return RB_OK;
}
