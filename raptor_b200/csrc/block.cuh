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

// ------------------------------------------------- 16-byte column groups --
// VW = 16 / sizeof(T) consecutive columns of one block-vector row move as one
// 16-byte access (float4 / double2).  The vectorised kernels give a lane VW
// columns of its row, so a warp covers VW times the rows of the
// one-column-a-lane layout per step and every load instruction moves four
// (FP32) or two (FP64) times the bytes: at k >= VW the block kernels are
// bound by the loads they keep in flight, not by their bytes.  Used when k is
// a multiple of VW and every vector the kernel touches starts on a 16-byte
// boundary (rows then start on one too).
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
    using type = float4;
    static constexpr int n = 4;
};
template <>
struct Vec16<double> {
    using type = double2;
    static constexpr int n = 2;
};

template <typename T, int VW>
__device__ __forceinline__ void vunpack(const typename Vec16<T>::type& u, T (&v)[VW]) {
    static_assert(VW == Vec16<T>::n, "16-byte groups");
    if constexpr (VW == 4) {
        v[0] = u.x; v[1] = u.y; v[2] = u.z; v[3] = u.w;
    } else {
        v[0] = u.x; v[1] = u.y;
    }
}
// through the read-only path (vectors no thread of the kernel writes)
template <typename T, int VW>
__device__ __forceinline__ void vload_ro(const T* p, T (&v)[VW]) {
    vunpack<T, VW>(__ldg(reinterpret_cast<const typename Vec16<T>::type*>(p)), v);
}
// a plain load (the thread may write the same entries afterwards)
template <typename T, int VW>
__device__ __forceinline__ void vload(const T* p, T (&v)[VW]) {
    vunpack<T, VW>(*reinterpret_cast<const typename Vec16<T>::type*>(p), v);
}
template <typename T, int VW>
__device__ __forceinline__ void vstore(T* p, const T (&v)[VW]) {
    static_assert(VW == Vec16<T>::n, "16-byte groups");
    typename Vec16<T>::type u;
    if constexpr (VW == 4) {
        u.x = v[0]; u.y = v[1]; u.z = v[2]; u.w = v[3];
    } else {
        u.x = v[0]; u.y = v[1];
    }
    *reinterpret_cast<typename Vec16<T>::type*>(p) = u;
}

inline bool al16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// ----------------------------------------------------------- epilogues --
// operator(): one entry (i, c); vec: the VW entries (i, c0 .. c0 + VW - 1),
// each computed as operator() computes it; al16: every vector starts on a
// 16-byte boundary.
template <typename TY>
struct BStore {
    TY* y;
    template <typename A>
    __device__ void operator()(long i, int c, int k, A s) const { y[i * k + c] = (TY)s; }
    template <int VW, typename A>
    __device__ void vec(long i, int c0, int k, const A (&s)[VW]) const {
        TY o[VW];
#pragma unroll
        for (int v = 0; v < VW; v++) o[v] = (TY)s[v];
        vstore<TY, VW>(y + i * k + c0, o);
    }
    bool al16v() const { return al16(y); }
};

template <typename TB, typename TY>
struct BResidual {
    const TB* b;
    TY* r;
    template <typename A>
    __device__ void operator()(long i, int c, int k, A s) const {
        r[i * k + c] = (TY)((A)b[i * k + c] - s);
    }
    template <int VW, typename A>
    __device__ void vec(long i, int c0, int k, const A (&s)[VW]) const {
        TB bb[VW];
        vload_ro<TB, VW>(b + i * k + c0, bb);
        TY o[VW];
#pragma unroll
        for (int v = 0; v < VW; v++) o[v] = (TY)((A)bb[v] - s[v]);
        vstore<TY, VW>(r + i * k + c0, o);
    }
    bool al16v() const { return al16(b) && al16(r); }
};

template <typename TY>
struct BAppend {
    TY* y;
    template <typename A>
    __device__ void operator()(long i, int c, int k, A s) const {
        y[i * k + c] = (TY)((A)y[i * k + c] + s);
    }
    template <int VW, typename A>
    __device__ void vec(long i, int c0, int k, const A (&s)[VW]) const {
        TY yy[VW];
        vload<TY, VW>(y + i * k + c0, yy);
#pragma unroll
        for (int v = 0; v < VW; v++) yy[v] = (TY)((A)yy[v] + s[v]);
        vstore<TY, VW>(y + i * k + c0, yy);
    }
    bool al16v() const { return al16(y); }
};

template <typename TY>
struct BAddTo {
    const TY* x0;
    TY* y;
    template <typename A>
    __device__ void operator()(long i, int c, int k, A s) const {
        y[i * k + c] = (TY)((A)x0[i * k + c] + s);
    }
    template <int VW, typename A>
    __device__ void vec(long i, int c0, int k, const A (&s)[VW]) const {
        TY xx[VW];
        vload_ro<TY, VW>(x0 + i * k + c0, xx);
#pragma unroll
        for (int v = 0; v < VW; v++) xx[v] = (TY)((A)xx[v] + s[v]);
        vstore<TY, VW>(y + i * k + c0, xx);
    }
    bool al16v() const { return al16(x0) && al16(y); }
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
    template <int VW, typename A>
    __device__ void vec(long i, int c0, int k, const A (&s)[VW]) const {
        const long e = i * k + c0;
        T xx[VW], bb[VW];
        vload_ro<T, VW>(xo + e, xx);
        vload_ro<T, VW>(b + e, bb);
        const A d = (A)__ldg(dinv + i);
        T o[VW];
#pragma unroll
        for (int v = 0; v < VW; v++) o[v] = (T)((A)xx[v] + d * ((A)bb[v] - s[v]));
        vstore<T, VW>(xn + e, o);
    }
    bool al16v() const { return al16(xo) && al16(b) && al16(xn); }
};

// ------------------------------------------------ per-column reductions --
// Each lane carries a partial for its column c = lane % KP.  The block sums
// them per column (warp shuffles over the row lanes, then the warps in a
// fixed order), writes partials[block * KP + c], and the last block to
// finish sums the block partials per column in a fixed order and calls
// fin(c, total) for c < k.  Bit-reproducible for a given grid.
// The block's per-warp column sums wpart[w][c] onwards.
template <int KP, class Fin>
__device__ void block_reduce_cols_tail(double (*wpart)[KP], int k, const ReduceSlot& rs, Fin fin) {
    constexpr int kWarps = 256 / 32;
    constexpr int kStrands = 256 / KP;
    __shared__ double spart[256];
    __shared__ bool is_last;
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

template <int KP, class Fin>
__device__ void block_reduce_cols(double v, int k, const ReduceSlot& rs, Fin fin) {
    constexpr int kWarps = 256 / 32;
    __shared__ double wpart[kWarps][KP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = KP; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane < KP) wpart[wid][lane] = v;
    block_reduce_cols_tail<KP>(wpart, k, rs, fin);
}

// The same with VW columns a lane: lane l carries columns (l % LPR) VW + v.
template <int LPR, int VW, class Fin>
__device__ void block_reduce_cols_v(double (&v)[VW], int k, const ReduceSlot& rs, Fin fin) {
    constexpr int KP = LPR * VW;
    constexpr int kWarps = 256 / 32;
    __shared__ double wpart[kWarps][KP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = LPR; o < 32; o <<= 1)
#pragma unroll
        for (int q = 0; q < VW; q++) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if (lane < LPR)
#pragma unroll
        for (int q = 0; q < VW; q++) wpart[wid][lane * VW + q] = v[q];
    block_reduce_cols_tail<KP>(wpart, k, rs, fin);
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

// ------------------------------------------------ vectorised CSR SpMM --
// LPR = KP / VW lanes a row, each with VW columns (Vec16); 32 / LPR rows a
// warp step.  The row's indices and values are broadcast loads (the LPR
// lanes of a row read the same entry); every lane then has the 16-byte
// gathers of up to RB_BLOCK_VEC_UN nonzeros in flight before it uses the
// first.  Each column's products are added in increasing position, as in
// k_csr_block with one row split.
#ifndef RB_BLOCK_VEC_UN
#define RB_BLOCK_VEC_UN 8
#endif

template <int LPR, typename TV, typename TX, typename Acc>
__device__ __forceinline__ void csr_row_v(int rs, int re, bool on, const int* __restrict__ ci,
                                          const TV* __restrict__ cv, const TX* __restrict__ X,
                                          int k, int c0, Acc (&acc)[Vec16<TX>::n]) {
    constexpr int VW = Vec16<TX>::n;
    constexpr int UN = RB_BLOCK_VEC_UN;
#pragma unroll
    for (int v = 0; v < VW; v++) acc[v] = Acc(0);
    for (int j = rs; j < re; j += UN) {
        int cc[UN];
        TV vv[UN];
#pragma unroll
        for (int u = 0; u < UN; u++) {
            const bool in = j + u < re;
            cc[u] = in ? __ldg(ci + j + u) : 0;
            vv[u] = in ? __ldg(cv + j + u) : TV(0);
        }
        TX xx[UN][VW];
#pragma unroll
        for (int u = 0; u < UN; u++) {
            if (on && j + u < re) {
                vload_ro<TX, VW>(X + (long)cc[u] * k + c0, xx[u]);
            } else {
#pragma unroll
                for (int v = 0; v < VW; v++) xx[u][v] = TX(0);
            }
        }
#pragma unroll
        for (int u = 0; u < UN; u++)
            if (j + u < re)
#pragma unroll
                for (int v = 0; v < VW; v++) acc[v] += (Acc)vv[u] * (Acc)xx[u][v];
    }
}

template <int LPR, typename TV, typename TX, typename Acc, class Epi>
__global__ void __launch_bounds__(256)
k_csr_block_v(long n, int k, const int* __restrict__ rp, const int* __restrict__ ci,
              const TV* __restrict__ cv, const TX* __restrict__ X, Epi epi) {
    constexpr int VW = Vec16<TX>::n;
    constexpr int RPW = 32 / LPR;
    const int lane = threadIdx.x & 31;
    const int c0 = (lane % LPR) * VW, sub = lane / LPR;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        const long row = base + sub;
        const bool on = row < n && c0 < k;
        int rs = 0, re = 0;
        if (row < n) { rs = __ldg(rp + row); re = __ldg(rp + row + 1); }
        Acc acc[VW];
        csr_row_v<LPR, TV, TX, Acc>(rs, re, on, ci, cv, X, k, c0, acc);
        if (on) epi.template vec<VW>(row, c0, k, acc);
    }
}

// Y = A P with the per-column dots p.y, VW columns a lane
template <int LPR, typename TV, class Fin>
__global__ void __launch_bounds__(256)
k_csr_block_dot_v(long n, int k, const int* __restrict__ rp, const int* __restrict__ ci,
                  const TV* __restrict__ cv, const double* __restrict__ P, double* __restrict__ Y,
                  ReduceSlot rsl, Fin fin) {
    constexpr int VW = Vec16<double>::n;
    constexpr int RPW = 32 / LPR;
    const int lane = threadIdx.x & 31;
    const int c0 = (lane % LPR) * VW, sub = lane / LPR;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    double red[VW];
#pragma unroll
    for (int v = 0; v < VW; v++) red[v] = 0.0;
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        const long row = base + sub;
        const bool on = row < n && c0 < k;
        int rs = 0, re = 0;
        if (row < n) { rs = __ldg(rp + row); re = __ldg(rp + row + 1); }
        double acc[VW];
        csr_row_v<LPR, TV, double, double>(rs, re, on, ci, cv, P, k, c0, acc);
        if (on) {
            double pp[VW];
            vload_ro<double, VW>(P + row * k + c0, pp);
            vstore<double, VW>(Y + row * k + c0, acc);
#pragma unroll
            for (int v = 0; v < VW; v++) red[v] += pp[v] * acc[v];
        }
    }
    block_reduce_cols_v<LPR, VW>(red, k, rsl, fin);
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

// ----------------------------------------------- vectorised DIA SpMM --
// LPR lanes a row with VW columns each (Vec16), 32 / LPR consecutive rows a
// warp step (their values of one diagonal share a 32-row slice); the
// diagonals are taken DC at a time, all values and 16-byte gathers of a
// group loaded before its products, which are added in diagonal order as
// in k_sdia_block.
template <int ND>
struct DiaChunk {
    static constexpr int DC = ND < 9 ? ND : 9;
    static_assert(ND % DC == 0, "diagonal groups");
};

template <int ND, int LPR, typename TV, typename TX, typename Acc>
__device__ __forceinline__ void sdia_row_v(long i, long n, bool on, const DiaOff& off,
                                           const TV* __restrict__ sv, const TX* __restrict__ X,
                                           int k, int c0, Acc (&acc)[Vec16<TX>::n]) {
    constexpr int VW = Vec16<TX>::n;
    constexpr int DC = DiaChunk<ND>::DC;
    const TV* a = sv + (i >> 5) * ND * 32 + (i & 31);
#pragma unroll
    for (int v = 0; v < VW; v++) acc[v] = Acc(0);
#pragma unroll
    for (int d0 = 0; d0 < ND; d0 += DC) {
        TV av[DC];
        TX xv[DC][VW];
#pragma unroll
        for (int d = 0; d < DC; d++) {
            const long j = i + off.o[d0 + d];
            const bool in = on && j >= 0 && j < n;
            av[d] = in ? __ldg(a + (d0 + d) * 32) : TV(0);
            if (in) {
                vload_ro<TX, VW>(X + j * k + c0, xv[d]);
            } else {
#pragma unroll
                for (int v = 0; v < VW; v++) xv[d][v] = TX(0);
            }
        }
#pragma unroll
        for (int d = 0; d < DC; d++)
#pragma unroll
            for (int v = 0; v < VW; v++) acc[v] += (Acc)av[d] * (Acc)xv[d][v];
    }
}

template <int ND, int LPR, typename TV, typename TX, typename Acc, class Epi>
__global__ void __launch_bounds__(256)
k_sdia_block_v(long n, int k, DiaOff off, const TV* __restrict__ sv, const TX* __restrict__ X,
               Epi epi) {
    constexpr int VW = Vec16<TX>::n;
    constexpr int RPW = 32 / LPR;
    const int lane = threadIdx.x & 31;
    const int c0 = (lane % LPR) * VW, sub = lane / LPR;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        const long i = base + sub;
        const bool on = i < n && c0 < k;
        Acc acc[VW];
        sdia_row_v<ND, LPR, TV, TX, Acc>(i, n, on, off, sv, X, k, c0, acc);
        if (on) epi.template vec<VW>(i, c0, k, acc);
    }
}

template <int ND, int LPR, typename TV, class Fin>
__global__ void __launch_bounds__(256)
k_sdia_block_dot_v(long n, int k, DiaOff off, const TV* __restrict__ sv,
                   const double* __restrict__ P, double* __restrict__ Y, ReduceSlot rsl, Fin fin) {
    constexpr int VW = Vec16<double>::n;
    constexpr int RPW = 32 / LPR;
    const int lane = threadIdx.x & 31;
    const int c0 = (lane % LPR) * VW, sub = lane / LPR;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    double red[VW];
#pragma unroll
    for (int v = 0; v < VW; v++) red[v] = 0.0;
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        const long i = base + sub;
        const bool on = i < n && c0 < k;
        double acc[VW];
        sdia_row_v<ND, LPR, TV, double, double>(i, n, on, off, sv, P, k, c0, acc);
        if (on) {
            double pp[VW];
            vload_ro<double, VW>(P + i * k + c0, pp);
            vstore<double, VW>(Y + i * k + c0, acc);
#pragma unroll
            for (int v = 0; v < VW; v++) red[v] += pp[v] * acc[v];
        }
    }
    block_reduce_cols_v<LPR, VW>(red, k, rsl, fin);
}

// ------------------------------------------------------- block BLAS-1 --
// x = dinv .* b per column (first Jacobi sweep from a zero guess)
// VW columns a thread (Vec16): thread t takes row t / LPR, columns
// (t % LPR) VW ..
template <int LPR, typename T>
__global__ void k_scale_first_block_v(long n, int k, const T* __restrict__ b,
                                      const T* __restrict__ dinv, T* __restrict__ x) {
    constexpr int VW = Vec16<T>::n;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long i = t / LPR;
    const int c0 = (int)(t % LPR) * VW;
    if (i >= n || c0 >= k) return;
    T bb[VW];
    vload_ro<T, VW>(b + i * k + c0, bb);
    const T d = __ldg(dinv + i);
#pragma unroll
    for (int v = 0; v < VW; v++) bb[v] = bb[v] * d;
    vstore<T, VW>(x + i * k + c0, bb);
}

// (thread t: row t / KP, column t % KP; no division by k per entry)
template <int KP, typename T>
__global__ void k_scale_first_block(long n, int k, const T* __restrict__ b,
                                    const T* __restrict__ dinv, T* __restrict__ x) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long i = t / KP;
    const int c = (int)(t % KP);
    if (i >= n || c >= k) return;
    const long e = i * k + c;
    x[e] = b[e] * dinv[i];
}

// Per-column dot a.b over n rows of k columns (FP64 accumulation; b FP64 or
// the FP32 output of a block cycle), through fin(c, t).
template <int KP, typename TB, class Fin>
__global__ void __launch_bounds__(256)
k_block_dot(long n, int k, const double* __restrict__ a, const TB* __restrict__ b,
            ReduceSlot rsl, Fin fin) {
    constexpr int RPW = 32 / KP;
    const int lane = threadIdx.x & 31;
    const int c = lane % KP, sub = lane / KP;
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    double t = 0.0;
    if (c < k)
        for (long i = gwarp * RPW + sub; i < n; i += nwarps * RPW)
            t += a[i * k + c] * (double)b[i * k + c];
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
// Lanes a row of the vectorised kernels (0: they do not apply): k a multiple
// of VW and every vector on a 16-byte boundary.
template <typename TX, class Epi>
int vec_lanes(int k, const TX* X, const Epi& epi) {
    constexpr int VW = Vec16<TX>::n;
    static const bool off = grid_per_sm("RAPTOR_B200_BLOCK_SCALAR", 0) > 0;
    if (off || k < VW || k % VW || !al16(X) || !epi.al16v()) return 0;
    return pow2_at_least(k) / VW;
}

#define RB_BLOCK_LPR_SWITCH(LPR, ...)                              \
    switch (LPR) {                                                  \
        case 1: { constexpr int kL = 1; __VA_ARGS__; } break;      \
        case 2: { constexpr int kL = 2; __VA_ARGS__; } break;      \
        case 4: { constexpr int kL = 4; __VA_ARGS__; } break;      \
        case 8: { constexpr int kL = 8; __VA_ARGS__; } break;      \
        default: { constexpr int kL = 16; __VA_ARGS__; } break;    \
    }

template <typename TV, typename TX, class Epi>
void launch_csr_block(const int* rp, const int* ci, const TV* cv, long n, int k, const TX* X,
                      Epi epi, int S) {
    if (n <= 0) return;
    using Acc = AccOf2<TV, TX>;
    if (const int lpr = vec_lanes(k, X, epi)) {
        RB_BLOCK_LPR_SWITCH(lpr, {
            auto kern = k_csr_block_v<kL, TV, TX, Acc, Epi>;
            const unsigned g = block_grid_gather((const void*)kern, n, kL, 1);
            kern<<<g, 256, 0, stream()>>>(n, k, rp, ci, cv, X, epi);
        });
        RB_CHECK_LAUNCH();
        return;
    }
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
    if (const int lpr = vec_lanes(k, P, BStore<double>{Y})) {
        RB_BLOCK_LPR_SWITCH(lpr, {
            auto kern = k_csr_block_dot_v<kL, TV, Fin>;
            const unsigned g = block_grid_gather((const void*)kern, n, kL, 1);
            ReduceSlot rs = global_reduce_slot((int)g * kMaxBlockK);
            kern<<<g, 256, 0, stream()>>>(n, k, rp, ci, cv, P, Y, rs, fin);
        });
        RB_CHECK_LAUNCH();
        return;
    }
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
    if (off.nd == 7 || off.nd == 27) {
        if (const int lpr = vec_lanes(k, X, epi)) {
            RB_BLOCK_LPR_SWITCH(lpr, {
                auto kern = off.nd == 7 ? k_sdia_block_v<7, kL, TV, TX, Acc, Epi>
                                        : k_sdia_block_v<27, kL, TV, TX, Acc, Epi>;
                const unsigned g = block_grid_gather((const void*)kern, n, kL, 1);
                kern<<<g, 256, 0, stream()>>>(n, k, off, sv, X, epi);
            });
            RB_CHECK_LAUNCH();
            return;
        }
    }
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
    if (off.nd == 7 || off.nd == 27) {
        if (const int lpr = vec_lanes(k, P, BStore<double>{Y})) {
            RB_BLOCK_LPR_SWITCH(lpr, {
                auto kern = off.nd == 7 ? k_sdia_block_dot_v<7, kL, TV, Fin>
                                        : k_sdia_block_dot_v<27, kL, TV, Fin>;
                const unsigned g = block_grid_gather((const void*)kern, n, kL, 1);
                ReduceSlot rs = global_reduce_slot((int)g * kMaxBlockK);
                kern<<<g, 256, 0, stream()>>>(n, k, off, sv, P, Y, rs, fin);
            });
            RB_CHECK_LAUNCH();
            return;
        }
    }
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

template <typename TB, class Fin>
void launch_block_dot(long n, int k, const double* a, const TB* b, Fin fin) {
    const int KP = pow2_at_least(k);
    const unsigned g = block_grid(n, KP, 1);
    ReduceSlot rs = global_reduce_slot((int)g * kMaxBlockK);
    RB_BLOCK_KP_SWITCH(KP, { k_block_dot<kKP, TB><<<g, 256, 0, stream()>>>(n, k, a, b, rs, fin); });
    RB_CHECK_LAUNCH();
}

}  // namespace rb
