// rb_common.cuh -- shared host/device infrastructure of libraptor_b200.
//
// Status codes, the per-thread last-error string, device buffers, the
// library stream, and warp-level helpers used by every kernel file.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/raptor_b200.h"

namespace rb {

// Error carried from deep inside the library to the C boundary.
struct Error : public std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

#define RB_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            throw ::rb::Error(e_ == cudaErrorMemoryAllocation ? RB_ERR_OOM : RB_ERR_CUDA, \
                              std::string(#call) + ": " + cudaGetErrorString(e_) +     \
                                  " at " + __FILE__ + ":" + std::to_string(__LINE__)); \
        }                                                                               \
    } while (0)

// Every kernel launch of the library is followed by RB_CHECK_LAUNCH, which
// also counts it (graph replays add their kernel-node count instead).
long long& launch_counter();
#define RB_CHECK_LAUNCH()                 \
    do {                                  \
        RB_CUDA(cudaGetLastError());      \
        ++::rb::launch_counter();         \
    } while (0)

#define RB_REQUIRE(cond, msg)                                  \
    do {                                                       \
        if (!(cond)) throw ::rb::Error(RB_ERR_INVALID, (msg)); \
    } while (0)

// The stream every library call is ordered on (set by rb_init / rb_set_stream).
cudaStream_t stream();
void set_stream(cudaStream_t s);
int sm_count();
// Blocks per SM a grid-stride kernel family is capped at: the value of the
// environment variable `env` when set to a positive integer, else `dflt`.
int grid_per_sm(const char* env, int dflt);
// Blocks of `threads` threads of kernel `fn` that fit on one SM at once
// (the occupancy calculator's answer, cached per kernel).
int resident_blocks_per_sm(const void* fn, int threads);

// Device allocations made through DevArray so far (every device buffer of
// the library is one); read through rb_device_alloc_count.
long long& device_alloc_counter();

// Owning device array (cudaMalloc'd; freed on destruction).
template <typename T>
struct DevArray {
    T* p = nullptr;
    size_t n = 0;
    DevArray() = default;
    explicit DevArray(size_t count) { alloc(count); }
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    DevArray(DevArray&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevArray& operator=(DevArray&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p; n = o.n; o.p = nullptr; o.n = 0;
        }
        return *this;
    }
    ~DevArray() { release(); }
    void alloc(size_t count) {
        release();
        n = count;
        if (count) {
            RB_CUDA(cudaMalloc(&p, sizeof(T) * count));
            ++::rb::device_alloc_counter();
        }
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void zero() {
        if (n) RB_CUDA(cudaMemsetAsync(p, 0, sizeof(T) * n, stream()));
    }
    void upload(const T* host, size_t count) {
        if (count) RB_CUDA(cudaMemcpyAsync(p, host, sizeof(T) * count, cudaMemcpyHostToDevice, stream()));
    }
    void download(T* host, size_t count) const {
        if (count) RB_CUDA(cudaMemcpyAsync(host, p, sizeof(T) * count, cudaMemcpyDeviceToHost, stream()));
    }
    std::vector<T> to_host() const {
        std::vector<T> h(n);
        download(h.data(), n);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return h;
    }
    T* get() const { return p; }
    size_t size() const { return n; }
};

template <typename T>
inline T read_scalar(const T* dev) {
    T h;
    RB_CUDA(cudaMemcpyAsync(&h, dev, sizeof(T), cudaMemcpyDeviceToHost, stream()));
    RB_CUDA(cudaStreamSynchronize(stream()));
    return h;
}

inline unsigned grid_for(long n, int block, long cap = 1L << 30) {
    long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

// ---------------------------------------------------------------- device --

__device__ __forceinline__ double warp_sum(double v, unsigned mask = 0xffffffffu) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(mask, v, o);
    return v;
}

template <int G, typename T>
__device__ __forceinline__ T group_sum(T v) {
    // sum over G consecutive lanes (G a power of two <= 32); result in every lane of the group
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
    return v;
}

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

}  // namespace rb
