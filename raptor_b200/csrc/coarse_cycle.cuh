// coarse_cycle.cuh -- the bottom of the V-cycle in one persistent launch.
//
// Below a few hundred thousand rows every operator of a level finishes in a
// couple of microseconds, so a kernel per operation is dominated by launch
// and drain latency.  Here all levels from l0 down to the coarsest run inside
// one cooperatively launched kernel: every block stays resident, walks the
// same sequence of row-parallel phases (pre-smooth, residual, restriction,
// ..., coarse LU solve, ..., prolongation, post-smooth) with grid-stride
// loops, and meets the others at a grid barrier between phases.
//
// The barrier spins with a bounded count: if it ever runs out (which a
// co-resident launch cannot cause) it raises an error flag, every block
// leaves, and the host reports the failure instead of hanging the GPU.
#pragma once

#include "spmv.cuh"

namespace rb {

template <typename T>
struct LevelDesc {
    int n, nc;
    const int* arp; const int* aci; const T* av; int gA;
    const int* prp; const int* pci; const T* pv; int gP;
    const int* rrp; const int* rci; const T* rv; int gR;
    const T* dinv;
    T* x; T* b; T* r; T* xt;
};

struct BarrierState {
    unsigned count;
    unsigned gen;
    int error;
    int pad;
};

constexpr long long kBarrierSpinLimit = 1LL << 24;   // ~seconds with nanosleep backoff

// Returns false once any block has flagged a timeout.
__device__ __forceinline__ bool grid_barrier(BarrierState* bs, unsigned nblocks) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &bs->gen;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&bs->count, 1u);
        if (arrived == nblocks - 1) {
            bs->count = 0;
            __threadfence();
            atomicAdd(&bs->gen, 1u);
        } else {
            long long spins = 0;
            while (*vgen == gen) {
                if (++spins > kBarrierSpinLimit || *(volatile int*)&bs->error) {
                    atomicExch(&bs->error, 1);
                    break;
                }
                if (spins > 4096) __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int*)&bs->error == 0;
}

// One row-parallel pass over all warps of the grid, G lanes per row (G is a
// runtime power of two; the shuffle width takes it directly).
template <typename T, class F>
__device__ __forceinline__ void grid_rows(int n, const int* __restrict__ rp,
                                          const int* __restrict__ ci, const T* __restrict__ cv,
                                          const T* __restrict__ x, int G, F f) {
    const int lane = threadIdx.x & 31;
    const int sub = lane / G, gl = lane & (G - 1);
    const int rpw = 32 / G;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long base = gwarp * rpw; base < n; base += nwarps * rpw) {
        const long row = base + sub;
        const bool valid = row < n;
        int s = 0, e = 0;
        if (valid) { s = rp[row]; e = rp[row + 1]; }
        T sum = 0;
        int j = s + gl;
        for (; j + 3 * G < e; j += 4 * G) {
            const int c0 = ci[j], c1 = ci[j + G], c2 = ci[j + 2 * G], c3 = ci[j + 3 * G];
            const T v0 = cv[j], v1 = cv[j + G], v2 = cv[j + 2 * G], v3 = cv[j + 3 * G];
            const T x0 = x[c0], x1 = x[c1], x2 = x[c2], x3 = x[c3];
            sum += v0 * x0;
            sum += v1 * x1;
            sum += v2 * x2;
            sum += v3 * x3;
        }
        for (; j < e; j += G) sum += cv[j] * x[ci[j]];
        for (int o = G >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, G);
        if (valid && gl == 0) f(row, sum);
    }
}

template <typename T>
__device__ __forceinline__ void grid_vec(int n, const T* b, const T* dinv, T* x) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        x[i] = b[i] * dinv[i];
}

// levels[0..nl-1] are l0..L-2 of the hierarchy; the coarsest system is the
// dense LU of size cn.  smooth: 0 none (the reference's Jacobi), 1 Jacobi-type.
constexpr int kFuseBlock = 1024;

template <typename T>
__global__ void __launch_bounds__(kFuseBlock)
k_coarse_cycle(const LevelDesc<T>* __restrict__ lv, int nl, const double* __restrict__ lu,
               const int* __restrict__ piv, int cn, T* xc, const T* bc, int smooth,
               BarrierState* bs) {
    extern __shared__ double y[];
    const unsigned nb = gridDim.x;
    // ---- down: pre-smooth from zero, residual, restriction
    for (int l = 0; l < nl; l++) {
        const LevelDesc<T> L = lv[l];
        if (smooth) {
            grid_vec<T>(L.n, L.b, L.dinv, L.x);
        } else {
            for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < L.n;
                 i += (long)gridDim.x * blockDim.x)
                L.x[i] = T(0);
        }
        if (!grid_barrier(bs, nb)) return;
        grid_rows<T>(L.n, L.arp, L.aci, L.av, L.x, L.gA,
                     [&](long i, T s) { L.r[i] = L.b[i] - s; });
        if (!grid_barrier(bs, nb)) return;
        T* bnext = (l + 1 < nl) ? lv[l + 1].b : const_cast<T*>(bc);
        grid_rows<T>(L.nc, L.rrp, L.rci, L.rv, L.r, L.gR, [&](long i, T s) { bnext[i] = s; });
        if (!grid_barrier(bs, nb)) return;
    }
    // ---- coarsest: LU of A_c^T (dgetrs 'N' on the row-major gather), block 0
    if (blockIdx.x == 0) {
        for (int i = threadIdx.x; i < cn; i += blockDim.x) y[i] = (double)bc[i];
        __syncthreads();
        if (threadIdx.x == 0)
            for (int k = 0; k < cn; k++) {
                int p = piv[k];
                if (p != k) { double t = y[k]; y[k] = y[p]; y[p] = t; }
            }
        __syncthreads();
        for (int j = 0; j < cn; j++) {
            const double yj = y[j];
            for (int i = j + 1 + threadIdx.x; i < cn; i += blockDim.x) y[i] -= lu[i + (size_t)j * cn] * yj;
            __syncthreads();
        }
        for (int j = cn - 1; j >= 0; j--) {
            if (threadIdx.x == 0) y[j] /= lu[j + (size_t)j * cn];
            __syncthreads();
            const double yj = y[j];
            for (int i = threadIdx.x; i < j; i += blockDim.x) y[i] -= lu[i + (size_t)j * cn] * yj;
            __syncthreads();
        }
        for (int i = threadIdx.x; i < cn; i += blockDim.x) xc[i] = (T)y[i];
    }
    if (!grid_barrier(bs, nb)) return;
    // ---- up: prolongation into xt, post-smooth back into x
    for (int l = nl - 1; l >= 0; l--) {
        const LevelDesc<T> L = lv[l];
        const T* xnext = (l + 1 < nl) ? lv[l + 1].x : xc;
        if (smooth) {
            grid_rows<T>(L.n, L.prp, L.pci, L.pv, xnext, L.gP,
                         [&](long i, T s) { L.xt[i] = L.x[i] + s; });
            if (!grid_barrier(bs, nb)) return;
            grid_rows<T>(L.n, L.arp, L.aci, L.av, L.xt, L.gA,
                         [&](long i, T s) { L.x[i] = L.xt[i] + L.dinv[i] * (L.b[i] - s); });
        } else {
            grid_rows<T>(L.n, L.prp, L.pci, L.pv, xnext, L.gP,
                         [&](long i, T s) { L.x[i] = L.x[i] + s; });
        }
        if (!grid_barrier(bs, nb)) return;
    }
}

}  // namespace rb
