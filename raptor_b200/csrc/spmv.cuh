// spmv.cuh -- CSR row kernels for the solve phase (HBM-bandwidth bound).
//
// One kernel template covers every "row of A times a vector, then something"
// operation of the V-cycle and the Krylov loop: b = A x (CSR_spmv,
// util/linalg/spmv.cpp:52-67), r = b - A x (CSR_residual, :69-85),
// b += A x (CSR_append, :88-103), a Jacobi sweep (par_relax.cpp:106-152), and
// b = A x fused with a deterministic dot product.  G lanes share a row; a
// warp walks 32/G consecutive rows per step so the column/value streams of
// neighbouring rows are read by one coalesced warp access, the gathered x
// goes through the read-only path, and partial sums meet in a shuffle tree.
#pragma once

#include <type_traits>

#include "rb_common.cuh"

namespace rb {

constexpr int kRowBlock = 256;

// Register budget of the CSR row kernels (minimum resident blocks per SM;
// 0 leaves the choice to the compiler).
#ifndef RB_ROWS_MINB
#define RB_ROWS_MINB 0
#endif
#if RB_ROWS_MINB > 0
#define RB_ROWS_BOUNDS __launch_bounds__(kRowBlock, RB_ROWS_MINB)
#else
#define RB_ROWS_BOUNDS __launch_bounds__(kRowBlock)
#endif

template <typename T> struct AccOf { using type = T; };
template <> struct AccOf<float> { using type = float; };
// Accumulator of a row product: the wider of the value and vector types
// (FP32 values against FP64 vectors accumulate in FP64).
template <typename TV, typename TX>
using AccOf2 = typename std::conditional<(sizeof(TX) > sizeof(TV)), TX, TV>::type;

// Block-level tree reduction followed by a fixed-order reduction of the block
// partials by the last block to finish; the result is bit-reproducible for a
// given grid.  fin(total) runs in one thread of the last block.
struct ReduceSlot {
    double* partials;   // gridDim.x entries
    unsigned* ticket;   // zero before the launch, reset by the last block
};

// Sum of p[first], p[first + step], ... below end, added in that order.  The
// loads bypass L1 (the values were written by other blocks) and are issued
// kReduceBatch at a time so that one round trip to L2 covers a batch.
constexpr int kReduceBatch = 16;
__device__ __forceinline__ double sum_strided_l2(const double* p, unsigned first, unsigned step,
                                                 unsigned end) {
    double t = 0.0;
    unsigned k = first;
    for (; k + (kReduceBatch - 1) * step < end; k += kReduceBatch * step) {
        double v[kReduceBatch];
#pragma unroll
        for (int u = 0; u < kReduceBatch; u++) v[u] = __ldcg(p + k + u * step);
#pragma unroll
        for (int u = 0; u < kReduceBatch; u++) t += v[u];
    }
    for (; k < end; k += step) t += __ldcg(p + k);
    return t;
}

template <class Fin>
__device__ void block_reduce_finish(double v, const ReduceSlot& rs, Fin fin) {
    __shared__ double warp_part[32];
    __shared__ bool is_last;
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) warp_part[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double t = lane < (int)(blockDim.x >> 5) ? warp_part[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) {
            rs.partials[blockIdx.x] = t;
            __threadfence();
            unsigned done = atomicAdd(rs.ticket, 1u);
            is_last = (done == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        // fixed-order second stage: thread k sums partials k, k+blockDim, ...
        // (loaded kReduceBatch at a time from L2, then added in order)
        double t = sum_strided_l2(rs.partials, threadIdx.x, blockDim.x, gridDim.x);
        t = warp_sum(t);
        if (lane == 0) warp_part[wid] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += warp_part[w];
            *rs.ticket = 0u;
            fin(tot);
        }
    }
}

// ------------------------------------------------------------ epilogues --
template <typename TY>
struct EpiStore {
    TY* y;
    template <typename A>
    __device__ void operator()(long i, A s, double&) const { y[i] = (TY)s; }
};

template <typename TB, typename TY>
struct EpiResidual {
    const TB* b;
    TY* r;
    template <typename A>
    __device__ void operator()(long i, A s, double&) const { r[i] = (TY)((A)b[i] - s); }
    // the same, split: operands loaded with the row's own loads, then applied
    struct Pre { TB b; };
    __device__ Pre pre(long i) const { return Pre{__ldg(b + i)}; }
    template <typename A>
    __device__ void post(long i, A s, double&, const Pre& p) const { r[i] = (TY)((A)p.b - s); }
};

template <typename TY>
struct EpiAppend {
    TY* y;
    template <typename A>
    __device__ void operator()(long i, A s, double&) const { y[i] = (TY)((A)y[i] + s); }
};

// y = x + P xc written to a second buffer (prolongation that also moves the
// iterate to the buffer the post-smoother should start from)
template <typename TY>
struct EpiAddTo {
    const TY* x0;
    TY* y;
    template <typename A>
    __device__ void operator()(long i, A s, double&) const { y[i] = (TY)((A)x0[i] + s); }
};

// Jacobi / L1-Jacobi: xn = xo + dinv (b - A xo); dinv already holds w/d_i.
template <typename TX, typename TB, typename TY>
struct EpiJacobi {
    const TX* xo;
    const TB* b;
    const TX* dinv;
    TY* xn;
    template <typename A>
    __device__ void operator()(long i, A s, double&) const {
        xn[i] = (TY)((A)xo[i] + (A)dinv[i] * ((A)b[i] - s));
    }
    struct Pre { TX xo; TB b; TX d; };
    __device__ Pre pre(long i) const { return Pre{__ldg(xo + i), __ldg(b + i), __ldg(dinv + i)}; }
    template <typename A>
    __device__ void post(long i, A s, double&, const Pre& p) const {
        xn[i] = (TY)((A)p.xo + (A)p.d * ((A)p.b - s));
    }
};

// Epilogues with a Pre type can load their per-row operands before the row's
// products (pre), and apply them after (post).
template <class Epi, class = void>
struct HasPre : std::false_type {};
template <class Epi>
struct HasPre<Epi, std::void_t<typename Epi::Pre>> : std::true_type {};

// The first Jacobi-type sweep from a zero iterate fused with the residual
// that follows it (ParMultilevel::cycle's relax then residual,
// par_multilevel.hpp:393-409, with x = 0 on entry): the sweep's result is
// x_i = b_i d_i (d = w / a_ii, or w / sum_j |a_ij| for L1-Jacobi), so the
// row product gathers b_j d_j in place of x_j, and the epilogue stores both
// x_i and r_i = b_i - (A x)_i.  Bit for bit what the sweep kernel and the
// residual kernel compute one after the other, in one pass instead of two:
// x is neither written before nor read back by the product.
template <typename T>
struct EpiFirstResidual {
    const T* b;
    const T* d;
    T* r;
    T* x;
    __host__ __device__ const T* gather_scale() const { return d; }
    template <typename A>
    __device__ void operator()(long i, A s, double&) const {
        const T bi = b[i];
        x[i] = (T)(bi * d[i]);
        r[i] = (T)((A)bi - s);
    }
    struct Pre { T b; T d; };
    __device__ Pre pre(long i) const { return Pre{__ldg(b + i), __ldg(d + i)}; }
    template <typename A>
    __device__ void post(long i, A s, double&, const Pre& p) const {
        x[i] = (T)(p.b * p.d);
        r[i] = (T)((A)p.b - s);
    }
};

// r = b - A x only when *gate is nonzero (read on the device when the kernel
// starts; otherwise every block returns at once).  Lets a step that only some
// iterations of a device-side loop need sit in the loop's graph.
template <typename TB, typename TY>
struct EpiResidualIf {
    const TB* b;
    TY* r;
    const int* gate;
    __device__ bool open() const { return *(volatile const int*)gate != 0; }
    template <typename A>
    __device__ void operator()(long i, A s, double&) const { r[i] = (TY)((A)b[i] - s); }
};

template <class Epi, class = void>
struct HasGate : std::false_type {};
template <class Epi>
struct HasGate<Epi, std::void_t<decltype(std::declval<const Epi&>().open())>> : std::true_type {};

// Epilogues with skip(base) let the strided row kernels pass over the rows
// [base, base + 32 / G) of a warp step without loading anything: an uneven
// batch's systems that have stopped (RowGate).  The answer must be the same
// for all rows of the step.  The blocked and shared-memory schedules are not
// compiled for such epilogues.
template <class Epi, class = void>
struct HasRowSkip : std::false_type {};
template <class Epi>
struct HasRowSkip<Epi, std::void_t<decltype(std::declval<const Epi&>().skip(0L))>>
    : std::true_type {};

// Rows per byte of a row gate (a multiple of every warp step's 32 / G rows,
// so that a step never straddles two bytes).
constexpr int kGateShift = 8;

// Epi restricted to the rows whose gate byte is zero: closed[row >> 8] != 0
// marks 256 rows that need no update.
template <class Epi>
struct RowGate : Epi {
    const unsigned char* closed;
    __device__ bool skip(long base) const { return closed[base >> kGateShift] != 0; }
};
template <class Epi>
RowGate<Epi> row_gate(const Epi& e, const unsigned char* closed) {
    return RowGate<Epi>{e, closed};
}

// Epilogues with gather_scale() make the row kernels gather x_j * scale_j.
template <class Epi, class = void>
struct ScaledGather : std::false_type {};
template <class Epi>
struct ScaledGather<Epi, std::void_t<decltype(std::declval<const Epi&>().gather_scale())>>
    : std::true_type {};

template <class Epi, typename TX>
__host__ __device__ inline const TX* gather_scale_of(const Epi& epi) {
    if constexpr (ScaledGather<Epi>::value) return epi.gather_scale();
    else return nullptr;
}

// y = A p and accumulate p.y (the CG denominator)
struct EpiStoreDot {
    const double* p;
    double* y;
    __device__ void operator()(long i, double s, double& red) const {
        y[i] = s;
        red += p[i] * s;
    }
};

unsigned row_grid_fwd(long n, int G);

struct NoFinish {
    __device__ void operator()(double) const {}
};

// ------------------------------------------------------------- kernels --
// Lanes per row G walk a row's nonzeros j = first, first + G, ...; a batch of
// RB_ROWS_BATCH of them per lane loads its column indices and values, then
// all of its gathers of x, then the products, so the gathers of a whole
// batch are in flight together (rows shorter than a batch predicate the
// rest off).  The products are added in increasing j, the same order as one
// nonzero at a time.  RB_ROWS_BATCH 0 keeps the older loop (four nonzeros
// ahead, then the tail one at a time).  Measured on the 192^3 FP32 cycle
// (levels 1-2, G = 8): batches of 4 cut the level-1 residual and sweep from
// 0.0698 to 0.0661 / 0.0677 ms and the cycle from 0.756 to 0.741 ms; batches
// of 8 were slower (0.0718 / 0.0885 ms).
#ifndef RB_ROWS_BATCH
#define RB_ROWS_BATCH 4
#endif

template <int G, int UN, typename Acc, bool SC = false, typename CI, typename TV, typename TX>
__device__ __forceinline__ Acc row_batched(int j, int e, const CI* __restrict__ ci,
                                           const TV* __restrict__ cv, const TX* __restrict__ xb,
                                           const TX* __restrict__ xsb = nullptr) {
    Acc sum = 0;
    for (; j < e; j += UN * G) {
        int cc[UN];
        TV vv[UN];
#pragma unroll
        for (int q = 0; q < UN; q++) {
            const bool ok = j + q * G < e;
            cc[q] = ok ? (int)__ldg(ci + j + q * G) : 0;
            vv[q] = ok ? __ldg(cv + j + q * G) : TV(0);
        }
        TX xx[UN];
#pragma unroll
        for (int q = 0; q < UN; q++) {
            if constexpr (SC)
                xx[q] = (j + q * G < e) ? (TX)(__ldg(xb + cc[q]) * __ldg(xsb + cc[q])) : TX(0);
            else
                xx[q] = (j + q * G < e) ? __ldg(xb + cc[q]) : TX(0);
        }
#pragma unroll
        for (int q = 0; q < UN; q++)
            if (j + q * G < e) sum += (Acc)vv[q] * (Acc)xx[q];
    }
    return sum;
}

template <int G, typename TV, typename TX, class Epi>
__global__ void RB_ROWS_BOUNDS
k_csr_rows(long n, const int* __restrict__ rp, const int* __restrict__ ci,
           const TV* __restrict__ cv, const TX* __restrict__ x, Epi epi) {
    using Acc = AccOf2<TV, TX>;
    constexpr bool SC = ScaledGather<Epi>::value;
    if constexpr (HasGate<Epi>::value) {
        if (!epi.open()) return;
    }
    const TX* xs = gather_scale_of<Epi, TX>(epi);
    constexpr int RPW = 32 / G;
    const int lane = threadIdx.x & 31;
    const int sub = lane / G, gl = lane & (G - 1);
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    double red = 0.0;
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        if constexpr (HasRowSkip<Epi>::value) {
            if (epi.skip(base)) continue;
        }
        const long row = base + sub;
        const bool valid = row < n;
        int s = 0, e = 0;
        if (valid) { s = __ldg(rp + row); e = __ldg(rp + row + 1); }
#if RB_ROWS_BATCH > 0
        Acc sum = row_batched<G, RB_ROWS_BATCH, Acc, SC>(s + gl, e, ci, cv, x, xs);
#else
        static_assert(!SC, "scaled gathers need the batched row loop");
        Acc sum = 0;
        int j = s + gl;
        // four independent index/value loads ahead of their gathers
        for (; j + 3 * G < e; j += 4 * G) {
            const int c0 = __ldg(ci + j), c1 = __ldg(ci + j + G);
            const int c2 = __ldg(ci + j + 2 * G), c3 = __ldg(ci + j + 3 * G);
            const TV v0 = __ldg(cv + j), v1 = __ldg(cv + j + G);
            const TV v2 = __ldg(cv + j + 2 * G), v3 = __ldg(cv + j + 3 * G);
            const TX x0 = __ldg(x + c0), x1 = __ldg(x + c1), x2 = __ldg(x + c2), x3 = __ldg(x + c3);
            sum += (Acc)v0 * (Acc)x0;
            sum += (Acc)v1 * (Acc)x1;
            sum += (Acc)v2 * (Acc)x2;
            sum += (Acc)v3 * (Acc)x3;
        }
        for (; j < e; j += G) sum += (Acc)__ldg(cv + j) * (Acc)__ldg(x + __ldg(ci + j));
#endif
        sum = group_sum<G>(sum);
        if (valid && gl == 0) epi(row, sum, red);
    }
    (void)red;
}

// The same row kernel over 16-bit column offsets: column = base[row] +
// c16[j].  For operators whose rows each span fewer than 65536 columns it
// reads 2 bytes of index per nonzero instead of 4 (FP32 values: 6 bytes per
// nonzero instead of 8).
template <int G, typename TV, typename TX, class Epi>
__global__ void RB_ROWS_BOUNDS
k_csr_rows16(long n, const int* __restrict__ rp, const int* __restrict__ rbase,
             const unsigned short* __restrict__ ci, const TV* __restrict__ cv,
             const TX* __restrict__ x, Epi epi) {
    using Acc = AccOf2<TV, TX>;
    constexpr bool SC = ScaledGather<Epi>::value;
    const TX* xs = gather_scale_of<Epi, TX>(epi);
    constexpr int RPW = 32 / G;
    const int lane = threadIdx.x & 31;
    const int sub = lane / G, gl = lane & (G - 1);
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    double red = 0.0;
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        if constexpr (HasRowSkip<Epi>::value) {
            if (epi.skip(base)) continue;
        }
        const long row = base + sub;
        const bool valid = row < n;
        int s = 0, e = 0, b0 = 0;
        if (valid) { s = __ldg(rp + row); e = __ldg(rp + row + 1); b0 = __ldg(rbase + row); }
        const TX* xb = x + b0;
#if RB_ROWS_BATCH > 0
        Acc sum = row_batched<G, RB_ROWS_BATCH, Acc, SC>(s + gl, e, ci, cv, xb,
                                                         SC ? xs + b0 : nullptr);
#else
        static_assert(!SC, "scaled gathers need the batched row loop");
        Acc sum = 0;
        int j = s + gl;
        for (; j + 3 * G < e; j += 4 * G) {
            const int c0 = __ldg(ci + j), c1 = __ldg(ci + j + G);
            const int c2 = __ldg(ci + j + 2 * G), c3 = __ldg(ci + j + 3 * G);
            const TV v0 = __ldg(cv + j), v1 = __ldg(cv + j + G);
            const TV v2 = __ldg(cv + j + 2 * G), v3 = __ldg(cv + j + 3 * G);
            const TX x0 = __ldg(xb + c0), x1 = __ldg(xb + c1), x2 = __ldg(xb + c2), x3 = __ldg(xb + c3);
            sum += (Acc)v0 * (Acc)x0;
            sum += (Acc)v1 * (Acc)x1;
            sum += (Acc)v2 * (Acc)x2;
            sum += (Acc)v3 * (Acc)x3;
        }
        for (; j < e; j += G) sum += (Acc)__ldg(cv + j) * (Acc)__ldg(xb + __ldg(ci + j));
#endif
        sum = group_sum<G>(sum);
        if (valid && gl == 0) epi(row, sum, red);
    }
    (void)red;
}

// The same row kernels with a blocked schedule: one block of
// kRowBlockBlk threads per SM, block b takes the contiguous rows
// [b R, (b + 1) R) and its warps walk them RPW rows at a time, so the
// columns an SM gathers stay within one window of x (a coarse operator's
// rows couple to neighbouring rows only) and its L1 serves the gathers that
// the strided schedule sends to L2.  Selected per operator by timing (the
// lanes-per-row value carries kRowsBlocked).
constexpr int kRowBlockBlk = 1024;
constexpr int kRowsBlocked = 64;

template <int G, typename TV, typename TX, class Epi>
__global__ void __launch_bounds__(kRowBlockBlk, 1)
k_csr_rows_blk(long n, const int* __restrict__ rp, const int* __restrict__ ci,
               const TV* __restrict__ cv, const TX* __restrict__ x, Epi epi) {
    using Acc = AccOf2<TV, TX>;
    constexpr bool SC = ScaledGather<Epi>::value;
    if constexpr (HasGate<Epi>::value) {
        if (!epi.open()) return;
    }
    const TX* xs = gather_scale_of<Epi, TX>(epi);
    constexpr int RPW = 32 / G;
    const int lane = threadIdx.x & 31;
    const int sub = lane / G, gl = lane & (G - 1);
    const long per = ((n + gridDim.x - 1) / gridDim.x + RPW - 1) / RPW * RPW;
    const long first = (long)blockIdx.x * per;
    const long last = first + per < n ? first + per : n;
    const int warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    double red = 0.0;
    for (long base = first + (long)warp * RPW; base < last; base += (long)nw * RPW) {
        const long row = base + sub;
        const bool valid = row < last;
        int s = 0, e = 0;
        if (valid) { s = __ldg(rp + row); e = __ldg(rp + row + 1); }
        Acc sum = row_batched<G, RB_ROWS_BATCH, Acc, SC>(s + gl, e, ci, cv, x, xs);
        sum = group_sum<G>(sum);
        if (valid && gl == 0) epi(row, sum, red);
    }
    (void)red;
}

template <int G, typename TV, typename TX, class Epi>
__global__ void __launch_bounds__(kRowBlockBlk, 1)
k_csr_rows16_blk(long n, const int* __restrict__ rp, const int* __restrict__ rbase,
                 const unsigned short* __restrict__ ci, const TV* __restrict__ cv,
                 const TX* __restrict__ x, Epi epi) {
    using Acc = AccOf2<TV, TX>;
    constexpr bool SC = ScaledGather<Epi>::value;
    const TX* xs = gather_scale_of<Epi, TX>(epi);
    constexpr int RPW = 32 / G;
    const int lane = threadIdx.x & 31;
    const int sub = lane / G, gl = lane & (G - 1);
    const long per = ((n + gridDim.x - 1) / gridDim.x + RPW - 1) / RPW * RPW;
    const long first = (long)blockIdx.x * per;
    const long last = first + per < n ? first + per : n;
    const int warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    double red = 0.0;
    for (long base = first + (long)warp * RPW; base < last; base += (long)nw * RPW) {
        const long row = base + sub;
        const bool valid = row < last;
        int s = 0, e = 0, b0 = 0;
        if (valid) { s = __ldg(rp + row); e = __ldg(rp + row + 1); b0 = __ldg(rbase + row); }
        Acc sum = row_batched<G, RB_ROWS_BATCH, Acc, SC>(s + gl, e, ci, cv, x + b0,
                                                         SC ? xs + b0 : nullptr);
        sum = group_sum<G>(sum);
        if (valid && gl == 0) epi(row, sum, red);
    }
    (void)red;
}

template <int G, typename TV, class Fin>
__global__ void RB_ROWS_BOUNDS
k_csr_rows_dot(long n, const int* __restrict__ rp, const int* __restrict__ ci,
               const TV* __restrict__ cv, const double* __restrict__ x, EpiStoreDot epi,
               ReduceSlot rs, Fin fin) {
    constexpr int RPW = 32 / G;
    const int lane = threadIdx.x & 31;
    const int sub = lane / G, gl = lane & (G - 1);
    const long gwarp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    double red = 0.0;
    for (long base = gwarp * RPW; base < n; base += nwarps * RPW) {
        const long row = base + sub;
        const bool valid = row < n;
        int s = 0, e = 0;
        if (valid) { s = __ldg(rp + row); e = __ldg(rp + row + 1); }
#if RB_ROWS_BATCH > 0
        double sum = row_batched<G, RB_ROWS_BATCH, double>(s + gl, e, ci, cv, x);
#else
        double sum = 0;
        int j = s + gl;
        for (; j + 3 * G < e; j += 4 * G) {
            const int c0 = __ldg(ci + j), c1 = __ldg(ci + j + G);
            const int c2 = __ldg(ci + j + 2 * G), c3 = __ldg(ci + j + 3 * G);
            const TV v0 = __ldg(cv + j), v1 = __ldg(cv + j + G);
            const TV v2 = __ldg(cv + j + 2 * G), v3 = __ldg(cv + j + 3 * G);
            const double x0 = __ldg(x + c0), x1 = __ldg(x + c1), x2 = __ldg(x + c2), x3 = __ldg(x + c3);
            sum += (double)v0 * x0;
            sum += (double)v1 * x1;
            sum += (double)v2 * x2;
            sum += (double)v3 * x3;
        }
        for (; j < e; j += G) sum += (double)__ldg(cv + j) * __ldg(x + __ldg(ci + j));
#endif
        sum = group_sum<G>(sum);
        if (valid && gl == 0) epi(row, sum, red);
    }
    block_reduce_finish(red, rs, fin);
}

ReduceSlot global_reduce_slot(int grid);

// y = A x fused with x.y (deterministic), CSR with values of type TV and
// FP64 vectors/accumulation.
template <typename TV, class Fin>
void launch_rows_dot(const int* rp, const int* ci, const TV* cv, long n, const double* x,
                     double* y, int G, Fin fin) {
    G &= kRowsBlocked - 1;   // the dot kernel runs the strided schedule only
    if (G <= 0) G = 8;
    const unsigned grid = row_grid_fwd(n, G);
    ReduceSlot rs = global_reduce_slot(grid);
    EpiStoreDot epi{x, y};
    switch (G) {
        case 1: k_csr_rows_dot<1, TV><<<grid, kRowBlock, 0, stream()>>>(n, rp, ci, cv, x, epi, rs, fin); break;
        case 2: k_csr_rows_dot<2, TV><<<grid, kRowBlock, 0, stream()>>>(n, rp, ci, cv, x, epi, rs, fin); break;
        case 4: k_csr_rows_dot<4, TV><<<grid, kRowBlock, 0, stream()>>>(n, rp, ci, cv, x, epi, rs, fin); break;
        case 8: k_csr_rows_dot<8, TV><<<grid, kRowBlock, 0, stream()>>>(n, rp, ci, cv, x, epi, rs, fin); break;
        case 16: k_csr_rows_dot<16, TV><<<grid, kRowBlock, 0, stream()>>>(n, rp, ci, cv, x, epi, rs, fin); break;
        default: k_csr_rows_dot<32, TV><<<grid, kRowBlock, 0, stream()>>>(n, rp, ci, cv, x, epi, rs, fin); break;
    }
    RB_CHECK_LAUNCH();
}

// Lanes per row from the mean row length (a power of two in 2..32).
inline int pick_group(long n, long long nnz) {
    double mean = n > 0 ? (double)nnz / (double)n : 1.0;
    if (mean <= 3) return 2;
    if (mean <= 6) return 4;
    if (mean <= 14) return 8;
    if (mean <= 40) return 16;
    return 32;
}

inline unsigned row_grid(long n, int G) {
    long warps = (n * G + 31) / 32;
    long blocks = (warps * 32 + kRowBlock - 1) / kRowBlock;
    static const int per_sm = grid_per_sm("RAPTOR_B200_GRID_ROWS", 16);
    long cap = (long)sm_count() * per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (unsigned)blocks;
}

inline unsigned row_grid_fwd(long n, int G) { return row_grid(n, G); }

template <typename TV, typename TX, class Epi>
void launch_rows(const int* rp, const int* ci, const TV* cv, long n, long long nnz, const TX* x,
                 Epi epi, int G = 0, cudaStream_t st = nullptr) {
    if (n <= 0) return;
    if (!st) st = stream();
    if (G <= 0) G = pick_group(n, nnz);
    if constexpr (HasRowSkip<Epi>::value) G &= kRowsBlocked - 1;
    else if (G & kRowsBlocked) {
        const unsigned g = (unsigned)sm_count();
        switch (G & (kRowsBlocked - 1)) {
            case 1: k_csr_rows_blk<1><<<g, kRowBlockBlk, 0, st>>>(n, rp, ci, cv, x, epi); break;
            case 2: k_csr_rows_blk<2><<<g, kRowBlockBlk, 0, st>>>(n, rp, ci, cv, x, epi); break;
            case 4: k_csr_rows_blk<4><<<g, kRowBlockBlk, 0, st>>>(n, rp, ci, cv, x, epi); break;
            case 8: k_csr_rows_blk<8><<<g, kRowBlockBlk, 0, st>>>(n, rp, ci, cv, x, epi); break;
            case 16: k_csr_rows_blk<16><<<g, kRowBlockBlk, 0, st>>>(n, rp, ci, cv, x, epi); break;
            default: k_csr_rows_blk<32><<<g, kRowBlockBlk, 0, st>>>(n, rp, ci, cv, x, epi); break;
        }
        RB_CHECK_LAUNCH();
        return;
    }
    const unsigned grid = row_grid(n, G);
    switch (G) {
        case 1: k_csr_rows<1><<<grid, kRowBlock, 0, st>>>(n, rp, ci, cv, x, epi); break;
        case 2: k_csr_rows<2><<<grid, kRowBlock, 0, st>>>(n, rp, ci, cv, x, epi); break;
        case 4: k_csr_rows<4><<<grid, kRowBlock, 0, st>>>(n, rp, ci, cv, x, epi); break;
        case 8: k_csr_rows<8><<<grid, kRowBlock, 0, st>>>(n, rp, ci, cv, x, epi); break;
        case 16: k_csr_rows<16><<<grid, kRowBlock, 0, st>>>(n, rp, ci, cv, x, epi); break;
        default: k_csr_rows<32><<<grid, kRowBlock, 0, st>>>(n, rp, ci, cv, x, epi); break;
    }
    RB_CHECK_LAUNCH();
}

template <typename TV, typename TX, class Epi>
void launch_rows16(const int* rp, const int* rbase, const unsigned short* c16, const TV* cv,
                   long n, long long nnz, const TX* x, Epi epi, int G = 0) {
    if (n <= 0) return;
    if (G <= 0) G = pick_group(n, nnz);
    cudaStream_t st = stream();
    if constexpr (HasRowSkip<Epi>::value) G &= kRowsBlocked - 1;
    else if (G & kRowsBlocked) {
        const unsigned g = (unsigned)sm_count();
        switch (G & (kRowsBlocked - 1)) {
            case 1: k_csr_rows16_blk<1><<<g, kRowBlockBlk, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
            case 2: k_csr_rows16_blk<2><<<g, kRowBlockBlk, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
            case 4: k_csr_rows16_blk<4><<<g, kRowBlockBlk, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
            case 8: k_csr_rows16_blk<8><<<g, kRowBlockBlk, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
            case 16: k_csr_rows16_blk<16><<<g, kRowBlockBlk, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
            default: k_csr_rows16_blk<32><<<g, kRowBlockBlk, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
        }
        RB_CHECK_LAUNCH();
        return;
    }
    const unsigned grid = row_grid(n, G);
    switch (G) {
        case 1: k_csr_rows16<1><<<grid, kRowBlock, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
        case 2: k_csr_rows16<2><<<grid, kRowBlock, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
        case 4: k_csr_rows16<4><<<grid, kRowBlock, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
        case 8: k_csr_rows16<8><<<grid, kRowBlock, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
        case 16: k_csr_rows16<16><<<grid, kRowBlock, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
        default: k_csr_rows16<32><<<grid, kRowBlock, 0, st>>>(n, rp, rbase, c16, cv, x, epi); break;
    }
    RB_CHECK_LAUNCH();
}

}  // namespace rb
