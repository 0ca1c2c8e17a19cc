// tail_cycle.cuh -- the bottom of the V-cycle in one launch of one cluster.
//
// Below some tens of thousands of rows every operator of a level is done in a
// few microseconds, and a kernel per operation costs a launch and a drain
// each.  Here all levels from the chosen one down to the coarsest run in a
// single launch of one thread-block cluster (up to 16 CTAs of 1024 threads,
// one per SM): the CTAs walk the same sequence of row-parallel phases
// (residual, restriction, ..., coarse solve, ..., prolongation, post-sweep)
// and meet at the hardware cluster barrier between phases
// (barrier.cluster.arrive.release / wait.acquire: no spinning, no counters in
// memory, so no wait can outlive the launch).  Vectors written inside the
// launch are read through L2 (ld.global.cg), so no CTA can see a stale L1 line.
//
// Each phase computes exactly what the separate kernels compute, in the same
// order (G lanes a row summing their nonzeros in increasing position, the
// same shuffle tree, the fused first sweep x = b d, the coarse product of
// k_coarse_mv), so the launch changes the time of a cycle, not its result.
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

constexpr int kTailBlock = 1024;
constexpr int kTailMaxCluster = 16;

__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// One row-parallel pass over every warp of the cluster, G lanes a row (G a
// runtime power of two), f(row, sum) by the row's first lane.  A lane takes
// its nonzeros kTailBatch at a time: the index and value loads of a batch,
// then all its gathers, then the products in increasing position (the order
// of the separate row kernel), so a warp keeps a batch of loads in flight
// instead of one dependent pair.  x was written in this launch: it is read
// through L2.
constexpr int kTailBatch = 4;
template <typename T, class F>
__device__ __forceinline__ void tail_rows(int n, const int* __restrict__ rp,
                                          const int* __restrict__ ci, const T* __restrict__ cv,
                                          const T* x, int G, F f) {
    const int lane = threadIdx.x & 31;
    const int sub = lane / G, gl = lane & (G - 1);
    const int rpw = 32 / G;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long base = gwarp * rpw; base < n; base += nwarps * rpw) {
        const long row = base + sub;
        const bool valid = row < n;
        int s = 0, e = 0;
        if (valid) { s = __ldg(rp + row); e = __ldg(rp + row + 1); }
        T sum = 0;
        for (int j = s + gl; j < e; j += kTailBatch * G) {
            int cc[kTailBatch];
            T vv[kTailBatch];
#pragma unroll
            for (int q = 0; q < kTailBatch; q++) {
                const bool ok = j + q * G < e;
                cc[q] = ok ? __ldg(ci + j + q * G) : 0;
                vv[q] = ok ? __ldg(cv + j + q * G) : T(0);
            }
            T xx[kTailBatch];
#pragma unroll
            for (int q = 0; q < kTailBatch; q++) xx[q] = (j + q * G < e) ? __ldcg(x + cc[q]) : T(0);
#pragma unroll
            for (int q = 0; q < kTailBatch; q++)
                if (j + q * G < e) sum += vv[q] * xx[q];
        }
        for (int o = G >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, G);
        if (valid && gl == 0) f(row, sum);
    }
}

// levels lv[0..nl-1] are the hierarchy's levels f..L-2; the coarsest system
// (cn rows) is solved with its explicit inverse cinv (column-major) when
// given, else with the LU factors (block 0 alone).  smooth: 1 one
// Jacobi-type sweep before and after the coarse correction, 0 none (the
// reference's Jacobi, which leaves x unchanged).
template <typename T>
__global__ void __launch_bounds__(kTailBlock, 1)
k_tail_cycle(const LevelDesc<T>* __restrict__ lv, int nl, const double* __restrict__ cinv,
             const double* __restrict__ lu, const int* __restrict__ piv, int cn, T* xc,
             const T* bc, int smooth) {
    extern __shared__ double y[];
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long nthreads = (long)gridDim.x * blockDim.x;
    // ---- first level: x = D^-1 b from zero (or x = 0)
    {
        const LevelDesc<T>& L = lv[0];
        for (long i = tid; i < L.n; i += nthreads)
            L.x[i] = smooth ? (T)(__ldcg(L.b + i) * __ldg(L.dinv + i)) : T(0);
    }
    // ---- down: residual, restriction (with the next level's first sweep)
    for (int l = 0; l < nl; l++) {
        const LevelDesc<T>& L = lv[l];
        cluster_barrier();
        tail_rows<T>(L.n, L.arp, L.aci, L.av, L.x, L.gA,
                     [&](long i, T s) { L.r[i] = (T)(__ldcg(L.b + i) - s); });
        cluster_barrier();
        const bool last = l + 1 == nl;
        T* bnext = last ? const_cast<T*>(bc) : lv[l + 1].b;
        T* xnext = last ? nullptr : lv[l + 1].x;
        const T* dnext = last ? nullptr : lv[l + 1].dinv;
        tail_rows<T>(L.nc, L.rrp, L.rci, L.rv, L.r, L.gR, [&](long i, T s) {
            bnext[i] = s;
            if (!last) xnext[i] = smooth ? (T)(s * __ldg(dnext + i)) : T(0);
        });
    }
    cluster_barrier();
    // ---- coarsest: x_c = A_c^-T b_c (the reference's dgetrs 'N' on its
    // row-major gather of A_c)
    if (cinv) {
        for (long i = tid; i < cn; i += nthreads) {
            double s = 0.0;
            for (int j = 0; j < cn; j++) s += cinv[(size_t)j * cn + i] * (double)__ldcg(bc + j);
            xc[i] = (T)s;
        }
    } else if (blockIdx.x == 0) {
        for (int i = threadIdx.x; i < cn; i += blockDim.x) y[i] = (double)__ldcg(bc + i);
        __syncthreads();
        if (threadIdx.x == 0)
            for (int k = 0; k < cn; k++) {
                const int p = piv[k];
                if (p != k) { const double t = y[k]; y[k] = y[p]; y[p] = t; }
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
    cluster_barrier();
    // ---- up: prolongation (into xt), post-sweep (back into x)
    for (int l = nl - 1; l >= 0; l--) {
        const LevelDesc<T>& L = lv[l];
        const T* xnext = (l + 1 < nl) ? lv[l + 1].x : xc;
        if (smooth) {
            tail_rows<T>(L.n, L.prp, L.pci, L.pv, xnext, L.gP,
                         [&](long i, T s) { L.xt[i] = (T)(__ldcg(L.x + i) + s); });
            cluster_barrier();
            tail_rows<T>(L.n, L.arp, L.aci, L.av, L.xt, L.gA, [&](long i, T s) {
                L.x[i] = (T)(__ldcg(L.xt + i) + __ldg(L.dinv + i) * (__ldcg(L.b + i) - s));
            });
        } else {
            tail_rows<T>(L.n, L.prp, L.pci, L.pv, xnext, L.gP,
                         [&](long i, T s) { L.x[i] = (T)(__ldcg(L.x + i) + s); });
        }
        if (l > 0) cluster_barrier();
    }
}

}  // namespace rb
