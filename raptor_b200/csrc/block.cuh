// block.cuh -- k right-hand sides at once: block-vector SpMM kernels.
//
// A block vector holds k columns interleaved by row: entry (i, c) at
// i * k + c.  One pass over A then serves all k columns: the values and
// column indices of a row are read once (a broadcast to the lanes of the
// row's columns), and the k entries of x at each column index are one
// contiguous run.  For a bandwidth-bound operator this divides the matrix
// traffic per right-hand side by k.
//
// Lane layout of a warp: KP lanes per row cover the columns (KP = k rounded
// up to a power of two; lanes c >= k idle), S such groups split the row's
// nonzeros, and 32 / (KP S) rows share the warp.  (KP, S) is the tile shape
// the autotuner picks per operator.
#pragma once

#include "dia.cuh"

namespace rb {

constexpr int kMaxBlockK = 32;

// Tuning knobs of the block kernels (loads in flight against occupancy).
// Measured on the SA 160^3 k = 8 / 32 solves: one row group per warp step
// for the diagonal kernels (U = 4 rows: 12.6 / 10.7 ms per right-hand side,
// U = 2: 9.86 / 7.96, U = 1: 9.41 / 6.78), the compiler's register choice
// (2 blocks per SM: 11.6 / 9.9), CSR rows staged through shared memory with
// up to 32 gathers per lane in flight (RB_BLOCK_CSR_STAGED, RB_BLOCK_STAGE_UN:
// k = 32 7.07 -> 6.64 ms per right-hand side together with grids of resident
// blocks only, against four index loads ahead of their gathers).
#ifndef RB_BLOCK_DIA_U
#define RB_BLOCK_DIA_U 1
#endif
#ifndef RB_BLOCK_MINB
#define RB_BLOCK_MINB 0
#endif
// Resident blocks per SM asked of the diagonal kernels with at most 9
// diagonals (0: the compiler's choice); wider stencils, and the kernel with
// the per-column dots at 32 columns, keep the compiler's choice.  Measured
// on the SA 160^3 solves, same box: 6 blocks 8.88 / 7.01 ms per right-hand
// side at k = 8 / 32, 8 blocks 9.39 / 7.05, compiler's choice (4 blocks, 64
// registers) 9.42 / 7.10; 6 blocks except for the dot kernel 9.41 / 6.69.
// The dot kernel alone (96^3, k = 32): 0.309 ms with 6 blocks (40
// registers), 0.200 ms with the compiler's 64 registers.
#ifndef RB_BLOCK_MINB_SMALL
#define RB_BLOCK_MINB_SMALL 6
#endif
#if RB_BLOCK_MINB > 0
#define RB_BLOCK_BOUNDS __launch_bounds__(256, RB_BLOCK_MINB)
#else
#define RB_BLOCK_BOUNDS \
    __launch_bounds__(256, (ND > 0 && ND <= 9 && RB_BLOCK_MINB_SMALL > 0) ? RB_BLOCK_MINB_SMALL : 1)
#endif

// ----------------------------------------------------------- epilogues --
template <typename TY>
struct BStore {
    TY* y;
    template <typename A>
    __device__ void operator()(long i, int c, int k, A s) const { y[i * k + c] = (TY)s; }
};

template <typename TB, typename TY>
struct BResidual {
    const TB* b;
    TY* r;
    template <typename A>
    __device__ void operator()(long i, int c, int k, A s) const {
        r[i * k + c] = (TY)((A)b[i * k + c] - s);
    }
};

template <typename TY>
struct BAppend {
    TY* y;
    template <typename A>
    __device__ void operator()(long i, int c, int k, A s) const {
        y[i * k + c] = (TY)((A)y[i * k + c] + s);
    }
};

template <typename TY>
struct BAddTo {
    const TY* x0;
    TY* y;
    template <typename A>
    __device__ void operator()(long i, int c, int k, A s) const {
        y[i * k + c] = (TY)((A)x0[i * k + c] + s);
    }
};

// xn = xo + dinv_i (b - A xo), dinv per row
template <typename T>
struct BJacobi {
    const T* xo;
    const T* b;
    const T* dinv;
    T* xn;
    template <typename A>
    __device__ void operator()(long i, int c, int k, A s) const {
        const long e = i * k + c;
        xn[e] = (T)((A)xo[e] + (A)dinv[i] * ((A)b[e] - s));
    }
};

// ------------------------------------------------ per-column reductions --
// Each lane carries a partial for its column c = lane % KP.  The block sums
// them per column (warp shuffles over the row lanes, then the warps in a
// fixed order), writes partials[block * KP + c], and the last block to
// finish sums the block partials per column in a fixed order and calls
// fin(c, total) for c < k.  Bit-reproducible for a given grid.
template <int KP, class Fin>
__device__ void block_reduce_cols(double v, int k, const ReduceSlot& rs, Fin fin) {
    constexpr int kWarps = 256 / 32;
    constexpr int kStrands = 256 / KP;
    __shared__ double wpart[kWarps][KP];
    __shared__ double spart[256];
    __shared__ bool is_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = KP; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane < KP) wpart[wid][lane] = v;
    __syncthreads();
    if (threadIdx.x < KP) {
        double t = 0.0;
        for (int w = 0; w < kWarps; w++) t += wpart[w][threadIdx.x];
        rs.partials[(size_t)blockIdx.x * KP + threadIdx.x] = t;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(rs.ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // strand q of column c sums blocks q, q + kStrands, ...
    const int c = threadIdx.x % KP, q = threadIdx.x / KP;
    // (block b's partial of column c sits at b * KP + c: strand q reads
    // indices (q + j kStrands) KP + c, j = 0, 1, ...)
    const double t = sum_strided_l2(rs.partials, (unsigned)(q * KP + c), (unsigned)(kStrands * KP),
                                    gridDim.x * (unsigned)KP);
    spart[threadIdx.x] = t;
    __syncthreads();
    if (threadIdx.x < KP) {
        double tot = 0.0;
        for (int s = 0; s < kStrands; s++) tot += spart[s * KP + threadIdx.x];
        if (threadIdx.x < k) fin(threadIdx.x, tot);
    }
    __syncthreads();
    if (threadIdx.x == 0) *rs.ticket = 0u;
}

// ----------------------------------------------------------- CSR SpMM --
#ifndef RB_BLOCK_CSR_STAGED
#define RB_BLOCK_CSR_STAGED 1
#endif

#ifndef RB_BLOCK_STAGE_UN
#define RB_BLOCK_STAGE_UN 32
#endif

#if RB_BLOCK_CSR_STAGED
// One row's sum for lane (c, s) of its row group, G = KP S lanes.  The group
// reads the row's column indices and values G at a time with one coalesced
// load into the warp's staging area (scol / sval, 32 entries per warp); split
// s then takes entries s KP .. s KP + KP - 1 of each chunk, and every lane
// issues the gathers of X for UN of them before it uses the first, so a
// row's gathers are in flight together instead of each waiting on its own
// index load.  nchunks is uniform over the warp (the longest row of the
// warp's groups): the staging area is shared by the whole warp.
template <int KP, int S, typename TV, typename TX, typename Acc>
__device__ __forceinline__ Acc staged_row(int rs, int re, int nchunks, const int* __restrict__ ci,
                                          const TV* __restrict__ cv, const TX* __restrict__ X,
                                          int k, int c, int s, int gl, int* scol, TV* sval) {
    constexpr int G = KP * S;
    constexpr int UN = KP >= RB_BLOCK_STAGE_UN ? RB_BLOCK_STAGE_UN : KP;
    Acc acc = 0;
    for (int ch = 0; ch < nchunks; ch++) {
        const int b0 = rs + ch * G;
        __syncwarp();
        if (b0 + gl < re) {
            scol[gl] = __ldg(ci + b0 + gl);
            sval[gl] = __ldg(cv + b0 + gl);
        }
        __syncwarp();
        const int cnt = min(max(re - b0 - s * KP, 0), KP);
        const int* pc = scol + s * KP;
        const TV* pv = sval + s * KP;
        if (c < k) {
            int u = 0;
            for (; u + UN <= cnt; u += UN) {
                TX xv[UN];
#pragma unroll
                for (int q = 0; q < UN; q++) xv[q] = __ldg(X + (long)pc[u + q] * k + c);
#pragma unroll
                for (int q = 0; q < UN; q++) acc += (Acc)pv[u + q] * (Acc)xv[q];
            }
            for (; u < cnt; u++) acc += (Acc)pv[u] * (Acc)__ldg(X + (long)pc[u] * k + c);
        }
    }
    return acc;
}
#endif

template <int KP, int S, typename TV, typename TX, typename Acc, class Epi>
__global__ void __launch_bounds__(256)
k_csr_block(long n, int k, const int* __restrict__ rp, const int* __restrict__ ci,
            const TV* __restrict__ cv, const TX* __restrict__ X, Epi epi) {
    constexpr int RPW = 32 / (KP * S);
    const int lane = threadIdx.x & 31;
    const int c = lane % KP, s = (lane / KP) % S, sub = lane / (KP * S);
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
#if RB_BLOCK_CSR_STAGED
    constexpr int G = KP * S;
    __shared__ __align__(16) int scol_all[8][32];
    __shared__ __align__(16) TV sval_all[8][32];
    int* scol = scol_all[threadIdx.x >> 5] + sub * G;
    TV* sval = sval_all[threadIdx.x >> 5] + sub * G;
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        const long row = base + sub;
        int rs = 0, re = 0;
        if (row < n) { rs = __ldg(rp + row); re = __ldg(rp + row + 1); }
        const int nch = __reduce_max_sync(0xffffffffu, (unsigned)((re - rs + G - 1) / G));
        Acc acc = staged_row<KP, S, TV, TX, Acc>(rs, re, nch, ci, cv, X, k, c, s, lane % G, scol, sval);
#else
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        const long row = base + sub;
        Acc acc = 0;
        if (row < n && c < k) {
            const int rs = __ldg(rp + row), re = __ldg(rp + row + 1);
            int j = rs + s;
            for (; j + 3 * S < re; j += 4 * S) {
                const int c0 = __ldg(ci + j), c1 = __ldg(ci + j + S);
                const int c2 = __ldg(ci + j + 2 * S), c3 = __ldg(ci + j + 3 * S);
                const TV v0 = __ldg(cv + j), v1 = __ldg(cv + j + S);
                const TV v2 = __ldg(cv + j + 2 * S), v3 = __ldg(cv + j + 3 * S);
                const TX x0 = __ldg(X + (long)c0 * k + c), x1 = __ldg(X + (long)c1 * k + c);
                const TX x2 = __ldg(X + (long)c2 * k + c), x3 = __ldg(X + (long)c3 * k + c);
                acc += (Acc)v0 * (Acc)x0;
                acc += (Acc)v1 * (Acc)x1;
                acc += (Acc)v2 * (Acc)x2;
                acc += (Acc)v3 * (Acc)x3;
            }
            for (; j < re; j += S) acc += (Acc)__ldg(cv + j) * (Acc)__ldg(X + (long)__ldg(ci + j) * k + c);
        }
#endif
#pragma unroll
        for (int o = KP; o < KP * S; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (row < n && c < k && s == 0) epi(row, c, k, acc);
    }
}

// Y = A P with the per-column dots p.y (FP64 vectors, values TV)
template <int KP, int S, typename TV, class Fin>
__global__ void __launch_bounds__(256)
k_csr_block_dot(long n, int k, const int* __restrict__ rp, const int* __restrict__ ci,
                const TV* __restrict__ cv, const double* __restrict__ P, double* __restrict__ Y,
                ReduceSlot rsl, Fin fin) {
    constexpr int RPW = 32 / (KP * S);
    const int lane = threadIdx.x & 31;
    const int c = lane % KP, s = (lane / KP) % S, sub = lane / (KP * S);
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    double red = 0.0;
#if RB_BLOCK_CSR_STAGED
    constexpr int G = KP * S;
    __shared__ __align__(16) int scol_all[8][32];
    __shared__ __align__(16) TV sval_all[8][32];
    int* scol = scol_all[threadIdx.x >> 5] + sub * G;
    TV* sval = sval_all[threadIdx.x >> 5] + sub * G;
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        const long row = base + sub;
        int rs = 0, re = 0;
        if (row < n) { rs = __ldg(rp + row); re = __ldg(rp + row + 1); }
        const int nch = __reduce_max_sync(0xffffffffu, (unsigned)((re - rs + G - 1) / G));
        double acc = staged_row<KP, S, TV, double, double>(rs, re, nch, ci, cv, P, k, c, s, lane % G,
                                                           scol, sval);
#else
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        const long row = base + sub;
        double acc = 0;
        if (row < n && c < k) {
            const int rs = __ldg(rp + row), re = __ldg(rp + row + 1);
            int j = rs + s;
            for (; j + 3 * S < re; j += 4 * S) {
                const int c0 = __ldg(ci + j), c1 = __ldg(ci + j + S);
                const int c2 = __ldg(ci + j + 2 * S), c3 = __ldg(ci + j + 3 * S);
                const double x0 = __ldg(P + (long)c0 * k + c), x1 = __ldg(P + (long)c1 * k + c);
                const double x2 = __ldg(P + (long)c2 * k + c), x3 = __ldg(P + (long)c3 * k + c);
                acc += (double)__ldg(cv + j) * x0;
                acc += (double)__ldg(cv + j + S) * x1;
                acc += (double)__ldg(cv + j + 2 * S) * x2;
                acc += (double)__ldg(cv + j + 3 * S) * x3;
            }
            for (; j < re; j += S) acc += (double)__ldg(cv + j) * __ldg(P + (long)__ldg(ci + j) * k + c);
        }
#endif
#pragma unroll
        for (int o = KP; o < KP * S; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (row < n && c < k && s == 0) {
            Y[row * k + c] = acc;
            red += P[row * k + c] * acc;
        }
    }
    block_reduce_cols<KP>(red, k, rsl, fin);
}

// ---------------------------------------------------- sliced DIA SpMM --
// A warp step covers U groups of 32 / KP consecutive rows; every value and
// gathered x of the step is loaded before the first product.
template <int ND>
struct DiaUnroll {
    static constexpr int U = (ND > 0 && ND <= 9) ? RB_BLOCK_DIA_U : 1;
};

template <int ND, int KP, typename TV, typename TX, typename Acc, class Epi>
__global__ void RB_BLOCK_BOUNDS
k_sdia_block(long n, int k, DiaOff off, const TV* __restrict__ sv, const TX* __restrict__ X,
             Epi epi) {
    constexpr int RPW = 32 / KP;
    constexpr int U = DiaUnroll<ND>::U;
    const int nd = ND > 0 ? ND : off.nd;
    const int lane = threadIdx.x & 31;
    const int c = lane % KP, sub = lane / KP;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long base = gwarp * RPW * U; base < n; base += nwarps * RPW * U) {
        if constexpr (ND > 0) {
            TV av[U][ND];
            TX xv[U][ND];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const long i = base + u * RPW + sub;
                const bool ok = i < n && c < k;
                const TV* a = sv + (i >> 5) * ND * 32 + (i & 31);
#pragma unroll
                for (int d = 0; d < ND; d++) {
                    const long j = i + off.o[d];
                    const bool in = ok && j >= 0 && j < n;
                    av[u][d] = in ? __ldg(a + d * 32) : TV(0);
                    xv[u][d] = in ? __ldg(X + j * k + c) : TX(0);
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const long i = base + u * RPW + sub;
                if (i >= n || c >= k) continue;
                Acc acc = 0;
#pragma unroll
                for (int d = 0; d < ND; d++) acc += (Acc)av[u][d] * (Acc)xv[u][d];
                epi(i, c, k, acc);
            }
        } else {
            const long i = base + sub;
            if (i >= n || c >= k) continue;
            const TV* a = sv + (i >> 5) * nd * 32 + (i & 31);
            Acc acc = 0;
            for (int d = 0; d < nd; d++) {
                const long j = i + off.o[d];
                if (j >= 0 && j < n) acc += (Acc)__ldg(a + d * 32) * (Acc)__ldg(X + j * k + c);
            }
            epi(i, c, k, acc);
        }
    }
}

template <int ND, int KP, typename TV, class Fin>
__global__ void __launch_bounds__(256, (ND > 0 && ND <= 9 && KP < 32 && RB_BLOCK_MINB_SMALL > 0)
                                           ? RB_BLOCK_MINB_SMALL : 1)
k_sdia_block_dot(long n, int k, DiaOff off, const TV* __restrict__ sv,
                 const double* __restrict__ P, double* __restrict__ Y, ReduceSlot rsl, Fin fin) {
    constexpr int RPW = 32 / KP;
    constexpr int U = DiaUnroll<ND>::U;
    const int nd = ND > 0 ? ND : off.nd;
    const int lane = threadIdx.x & 31;
    const int c = lane % KP, sub = lane / KP;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    double red = 0.0;
    for (long base = gwarp * RPW * U; base < n; base += nwarps * RPW * U) {
        if constexpr (ND > 0) {
            TV av[U][ND];
            double xv[U][ND];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const long i = base + u * RPW + sub;
                const bool ok = i < n && c < k;
                const TV* a = sv + (i >> 5) * ND * 32 + (i & 31);
#pragma unroll
                for (int d = 0; d < ND; d++) {
                    const long j = i + off.o[d];
                    const bool in = ok && j >= 0 && j < n;
                    av[u][d] = in ? __ldg(a + d * 32) : TV(0);
                    xv[u][d] = in ? __ldg(P + j * k + c) : 0.0;
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const long i = base + u * RPW + sub;
                if (i >= n || c >= k) continue;
                double acc = 0;
#pragma unroll
                for (int d = 0; d < ND; d++) acc += (double)av[u][d] * xv[u][d];
                Y[i * k + c] = acc;
                red += P[i * k + c] * acc;
            }
        } else {
            const long i = base + sub;
            if (i >= n || c >= k) continue;
            const TV* a = sv + (i >> 5) * nd * 32 + (i & 31);
            double acc = 0;
            for (int d = 0; d < nd; d++) {
                const long j = i + off.o[d];
                if (j >= 0 && j < n) acc += (double)__ldg(a + d * 32) * __ldg(P + j * k + c);
            }
            Y[i * k + c] = acc;
            red += P[i * k + c] * acc;
        }
    }
    block_reduce_cols<KP>(red, k, rsl, fin);
}

// ------------------------------------------------------- block BLAS-1 --
// x = dinv .* b per column (first Jacobi sweep from a zero guess)
template <typename T>
__global__ void k_scale_first_block(long n, int k, const T* __restrict__ b,
                                    const T* __restrict__ dinv, T* __restrict__ x) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n * k) x[e] = b[e] * dinv[e / k];
}

// Per-column dot a.b over n rows of k columns (FP64), through fin(c, t).
template <int KP, class Fin>
__global__ void __launch_bounds__(256)
k_block_dot(long n, int k, const double* __restrict__ a, const double* __restrict__ b,
            ReduceSlot rsl, Fin fin) {
    constexpr int RPW = 32 / KP;
    const int lane = threadIdx.x & 31;
    const int c = lane % KP, sub = lane / KP;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    double t = 0.0;
    if (c < k)
        for (long i = gwarp * RPW + sub; i < n; i += nwarps * RPW) t += a[i * k + c] * b[i * k + c];
    block_reduce_cols<KP>(t, k, rsl, fin);
}

// Coarsest level, k right-hand sides: one CTA per column.
template <typename T>
__global__ void k_lu_solve_block(int n, int k, const double* __restrict__ lu,
                                 const int* __restrict__ piv, const T* __restrict__ b,
                                 T* __restrict__ x) {
    extern __shared__ double y[];
    const int c = blockIdx.x;
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = (double)b[(long)i * k + c];
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
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[(long)i * k + c] = (T)y[i];
}

// ------------------------------------------------------------ launchers --
inline int pow2_at_least(int k) {
    int p = 1;
    while (p < k) p <<= 1;
    return p;
}

// Grid of a streaming kernel (no gathers): up to 16 blocks per SM.
inline unsigned block_grid(long n, int KP, int S) {
    const long rows_per_warp = 32 / (KP * S);
    long warps = (n + rows_per_warp - 1) / rows_per_warp;
    long blocks = (warps * 32 + 255) / 256;
    static const int per_sm = grid_per_sm("RAPTOR_B200_GRID_BLOCK", 16);
    long cap = std::min<long>((long)sm_count() * per_sm, 65536 / kMaxBlockK);
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (unsigned)blocks;
}

// Grid of a gathering SpMM kernel: only as many blocks as are resident at
// once, so that the warps in flight walk the rows as one contiguous window
// (row = step * resident warps + warp).  The k columns of the rows a window
// gathers from (its stencil or coarse-grid neighbours) are then read from
// HBM once and reused from L2; with more blocks than fit, the later waves
// revisit every neighbourhood after L2 has lost it, and a block vector of
// hundreds of MB is read two to three times per product.
inline unsigned block_grid_gather(const void* fn, long n, int KP, int S) {
    static const bool wide = grid_per_sm("RAPTOR_B200_BLOCK_WIDE", 0) > 0;
    if (wide) return block_grid(n, KP, S);
    const long rows_per_warp = 32 / (KP * S);
    long warps = (n + rows_per_warp - 1) / rows_per_warp;
    long blocks = (warps * 32 + 255) / 256;
    long cap = std::min<long>((long)sm_count() * resident_blocks_per_sm(fn, 256), 65536 / kMaxBlockK);
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (unsigned)blocks;
}

#define RB_BLOCK_KP_SWITCH(KP, ...)                     \
    switch (KP) {                                       \
        case 2: { constexpr int kKP = 2; __VA_ARGS__; } break;   \
        case 4: { constexpr int kKP = 4; __VA_ARGS__; } break;   \
        case 8: { constexpr int kKP = 8; __VA_ARGS__; } break;   \
        case 16: { constexpr int kKP = 16; __VA_ARGS__; } break; \
        default: { constexpr int kKP = 32; __VA_ARGS__; } break; \
    }

// CSR SpMM with tile shape (KP from k, S rows splits).
template <typename TV, typename TX, class Epi>
void launch_csr_block(const int* rp, const int* ci, const TV* cv, long n, int k, const TX* X,
                      Epi epi, int S) {
    if (n <= 0) return;
    using Acc = AccOf2<TV, TX>;
    const int KP = pow2_at_least(k);
    if (KP * S > 32) S = 32 / KP;
    auto go = [&](auto kern, int s) {
        const unsigned g = block_grid_gather((const void*)kern, n, KP, s);
        kern<<<g, 256, 0, stream()>>>(n, k, rp, ci, cv, X, epi);
    };
    RB_BLOCK_KP_SWITCH(KP, {
        if constexpr (kKP <= 8) {
            if (S >= 4) go(k_csr_block<kKP, 4, TV, TX, Acc, Epi>, 4);
            else if (S == 2) go(k_csr_block<kKP, 2, TV, TX, Acc, Epi>, 2);
            else go(k_csr_block<kKP, 1, TV, TX, Acc, Epi>, 1);
        } else if constexpr (kKP == 16) {
            if (S >= 2) go(k_csr_block<16, 2, TV, TX, Acc, Epi>, 2);
            else go(k_csr_block<16, 1, TV, TX, Acc, Epi>, 1);
        } else {
            go(k_csr_block<32, 1, TV, TX, Acc, Epi>, 1);
        }
    });
    RB_CHECK_LAUNCH();
}

template <typename TV, class Fin>
void launch_csr_block_dot(const int* rp, const int* ci, const TV* cv, long n, int k,
                          const double* P, double* Y, int S, Fin fin) {
    const int KP = pow2_at_least(k);
    if (KP * S > 32) S = 32 / KP;
    auto go = [&](auto kern, int s) {
        const unsigned g = block_grid_gather((const void*)kern, n, KP, s);
        ReduceSlot rs = global_reduce_slot((int)g * kMaxBlockK);
        kern<<<g, 256, 0, stream()>>>(n, k, rp, ci, cv, P, Y, rs, fin);
    };
    RB_BLOCK_KP_SWITCH(KP, {
        if constexpr (kKP <= 8) {
            if (S >= 4) go(k_csr_block_dot<kKP, 4, TV, Fin>, 4);
            else if (S == 2) go(k_csr_block_dot<kKP, 2, TV, Fin>, 2);
            else go(k_csr_block_dot<kKP, 1, TV, Fin>, 1);
        } else if constexpr (kKP == 16) {
            if (S >= 2) go(k_csr_block_dot<16, 2, TV, Fin>, 2);
            else go(k_csr_block_dot<16, 1, TV, Fin>, 1);
        } else {
            go(k_csr_block_dot<32, 1, TV, Fin>, 1);
        }
    });
    RB_CHECK_LAUNCH();
}

template <typename TV, typename TX, class Epi>
void launch_dia_block(const DiaOff& off, const TV* sv, long n, int k, const TX* X, Epi epi) {
    if (n <= 0) return;
    using Acc = AccOf2<TV, TX>;
    const int KP = pow2_at_least(k);
    auto go = [&](auto kern) {
        const unsigned g = block_grid_gather((const void*)kern, n, KP, 1);
        kern<<<g, 256, 0, stream()>>>(n, k, off, sv, X, epi);
    };
    RB_BLOCK_KP_SWITCH(KP, {
        switch (off.nd) {
            case 7: go(k_sdia_block<7, kKP, TV, TX, Acc, Epi>); break;
            case 27: go(k_sdia_block<27, kKP, TV, TX, Acc, Epi>); break;
            default: go(k_sdia_block<0, kKP, TV, TX, Acc, Epi>); break;
        }
    });
    RB_CHECK_LAUNCH();
}

template <typename TV, class Fin>
void launch_dia_block_dot(const DiaOff& off, const TV* sv, long n, int k, const double* P,
                          double* Y, Fin fin) {
    const int KP = pow2_at_least(k);
    auto go = [&](auto kern) {
        const unsigned g = block_grid_gather((const void*)kern, n, KP, 1);
        ReduceSlot rs = global_reduce_slot((int)g * kMaxBlockK);
        kern<<<g, 256, 0, stream()>>>(n, k, off, sv, P, Y, rs, fin);
    };
    RB_BLOCK_KP_SWITCH(KP, {
        switch (off.nd) {
            case 7: go(k_sdia_block_dot<7, kKP, TV, Fin>); break;
            case 27: go(k_sdia_block_dot<27, kKP, TV, Fin>); break;
            default: go(k_sdia_block_dot<0, kKP, TV, Fin>); break;
        }
    });
    RB_CHECK_LAUNCH();
}

template <class Fin>
void launch_block_dot(long n, int k, const double* a, const double* b, Fin fin) {
    const int KP = pow2_at_least(k);
    const unsigned g = block_grid(n, KP, 1);
    ReduceSlot rs = global_reduce_slot((int)g * kMaxBlockK);
    RB_BLOCK_KP_SWITCH(KP, { k_block_dot<kKP><<<g, 256, 0, stream()>>>(n, k, a, b, rs, fin); });
    RB_CHECK_LAUNCH();
}

}  // namespace rb
