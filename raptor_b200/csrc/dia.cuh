// dia.cuh -- sliced diagonal (stencil) storage for structured-grid levels.
//
// A matrix whose nonzeros lie on at most kMaxDiag distinct diagonals (every
// stencil_grid matrix: 9 for the 2D rotated diffusion, 27 for the 3D
// Laplacian) needs no column indices: a(i, i + off[d]).  Rows are grouped in
// slices of 32 (one warp) and a slice stores its nd coefficient columns one
// after another, vals[(slice * nd + d) * 32 + lane], zero where the stencil
// leaves the grid.  A warp therefore reads nd consecutive, 128-byte aligned
// lines (one L1 wavefront and one DRAM stream per warp) and gathers x at
// i + off[d], shifted contiguous runs that L1/L2 reuse across diagonals.
// For the 27-point operator an FP32 pass moves 108 instead of 216 bytes per
// row, and measured 0.19 ms against 0.32 ms for CSR on 192^3.
#pragma once

#include "spmv.cuh"

namespace rb {

constexpr int kMaxDiag = 32;

// Register budget of the diagonal kernels: at least RB_DIA_MINB blocks of
// 256 threads resident per SM (4: at most 64 registers a thread), with a row's
// values and gathered x loaded before the products (RB_DIA_TWO_PHASE) so a
// warp keeps its loads in flight.  Measured on 192^3 (27 diagonals, FP32
// values): the outer A p with FP64 vectors 0.222 -> 0.167 ms and the FP32
// residual 0.156 -> 0.151 ms against the compiler's default (32 registers,
// loads interleaved with the products); with 1 block a SM (up to 255
// registers) the kernels lose their occupancy and run at half speed.
#ifndef RB_DIA_MINB
#define RB_DIA_MINB 4
#endif
// The kernels without a dot (stores, residuals, sweeps) run one 32-row slice
// per warp (grid cap RB_DIA_GRID_ROWS blocks per SM, far above the slices of
// any level) with at least 3 resident blocks (85 registers); the dot kernel,
// whose last block sums one partial per block, keeps 32 blocks per SM and 4
// resident blocks.  Measured on 192^3 (27 diagonals, FP32 values): residual
// / Jacobi sweep 0.1516 / 0.1561 ms with (4 blocks, 32 per SM), 0.1498 /
// 0.1556 with (3, 32), 0.1496 / 0.1538 with (4, 64), 0.1455 / 0.1497 with
// (3, 128), 0.1435 / 0.1478 with (3, one slice per warp), 0.1681 / 0.1986
// with (2, one slice per warp); the dot kernel with 3 resident blocks 0.180
// against 0.166 ms.
#ifndef RB_DIA_MINB_ROWS
#define RB_DIA_MINB_ROWS 3
#endif
#ifndef RB_DIA_GRID_ROWS
#define RB_DIA_GRID_ROWS 1024
#endif
#ifndef RB_DIA_GRID_DOT
#define RB_DIA_GRID_DOT 32
#endif
#ifndef RB_DIA_TWO_PHASE
#define RB_DIA_TWO_PHASE 1
#endif
// Epilogue operands (b, the inverse diagonal, the old iterate) loaded with
// the row's own loads instead of after its products: level-0 FP32 Jacobi
// sweep on 192^3 0.158 -> 0.156 ms.
#ifndef RB_DIA_EPI_PREFETCH
#define RB_DIA_EPI_PREFETCH 1
#endif

// Offsets of the diagonals; with mask set, the operator has constant
// coefficients: every nonzero of diagonal d equals c[d], and bit d of
// mask[i] says whether a(i, i + o[d]) is nonzero.  The kernels then read 4
// bytes a row instead of nd values (the stored values stay for the kernels
// that do not take this form).  The same products in the same order: the
// results are those of the stored values bit for bit.
struct DiaOff {
    int nd;
    long long o[kMaxDiag];
    const unsigned* mask;
    double c[kMaxDiag];
    float cf[kMaxDiag];   // c in FP32 (exact: an FP32 level's values are FP32)
    // box-grid form (grid.cuh; needs mask): the stencil shape (GridShape,
    // 0 = none), the box nx x ny x nz (rows x fastest), planes per block and
    // rows in x a thread
    int grid, nx, ny, nz, gzc, gvx;
};

// *p through the read-only path when `on`, else 0, as one predicated load
// (the compiler otherwise branches around each conditional load; a diagonal
// a row, those branches saturated the SM's branch unit).  p is only formed,
// never read, when `on` is false.
__device__ __forceinline__ float ldg_if(const float* p, bool on) {
    float v;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\tmov.b32 %0, 0;\n\t"
        "@q ld.global.nc.f32 %0, [%1];\n\t}"
        : "=f"(v) : "l"(p), "r"((unsigned)on));
    return v;
}
__device__ __forceinline__ double ldg_if(const double* p, bool on) {
    double v;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\tmov.b64 %0, 0;\n\t"
        "@q ld.global.nc.f64 %0, [%1];\n\t}"
        : "=d"(v) : "l"(p), "r"((unsigned)on));
    return v;
}

// Coefficient d of a constant-coefficient operator in the value type TV (no
// conversion instruction for FP32 levels).
template <typename TV>
__device__ __forceinline__ TV dia_coef(const DiaOff& off, int d) {
    if constexpr (std::is_same<TV, float>::value) return off.cf[d];
    else return (TV)off.c[d];
}

}  // namespace rb

#include "grid.cuh"

namespace rb {

// SC: the gathered vector is x_j * xs_j (the fused first sweep, spmv.cuh);
// CC: constant coefficients (off.mask, off.c; base unused)
template <int ND, typename TV, typename TX, typename Acc, bool SC = false, bool CC = false>
__device__ __forceinline__ Acc sdia_row(long i, long n, const DiaOff& off, const TV* __restrict__ base,
                                        const TX* __restrict__ x,
                                        const TX* __restrict__ xs = nullptr) {
    Acc s = 0;
    if constexpr (ND > 0) {
#if RB_DIA_TWO_PHASE
        // all loads first (values, then the gathered x), then the products:
        // the warp keeps 2 ND loads in flight instead of waiting on each
        if constexpr (CC) {
            // a set mask bit implies 0 <= i + o[d] < n; a clear one is an entry
            // that is zero, whose product c_d * 0 adds nothing, as 0 * x does
            // FP32 vectors: one predicated load a diagonal (ldg_if).  FP64
            // vectors keep the compiler's conditional loads: with 27
            // predicated FP64 loads in flight the kernel spills (measured
            // 0.184 against 0.129 ms for the outer A p at 192^3).
            const unsigned m = i < n ? __ldg(off.mask + i) : 0u;
            TX xv[ND];
#pragma unroll
            for (int d = 0; d < ND; d++) {
                const bool on = (m >> d) & 1u;
                if constexpr (sizeof(TX) == 4) {
                    xv[d] = ldg_if(x + i + off.o[d], on);
                    if constexpr (SC) xv[d] = (TX)(xv[d] * ldg_if(xs + i + off.o[d], on));
                } else {
                    xv[d] = on ? __ldg(x + i + off.o[d]) : TX(0);
                    if constexpr (SC) xv[d] = on ? (TX)(xv[d] * __ldg(xs + i + off.o[d])) : TX(0);
                }
            }
            // (the coefficient in the accumulation type: the FP32 value
            // widened at setup, no conversion instruction a diagonal)
#pragma unroll
            for (int d = 0; d < ND; d++) s += dia_coef<Acc>(off, d) * (Acc)xv[d];
            return s;
        }
        TV v[ND];
        TX xv[ND];
#pragma unroll
        for (int d = 0; d < ND; d++) v[d] = __ldg(base + d * 32);
#pragma unroll
        for (int d = 0; d < ND; d++) {
            const long j = i + off.o[d];
            if constexpr (SC)
                xv[d] = (j >= 0 && j < n) ? (TX)(__ldg(x + j) * __ldg(xs + j)) : TX(0);
            else
                xv[d] = (j >= 0 && j < n) ? __ldg(x + j) : TX(0);
        }
#pragma unroll
        for (int d = 0; d < ND; d++) s += (Acc)v[d] * (Acc)xv[d];
#else
        static_assert(!SC && !CC, "scaled gathers and constant coefficients need the two-phase row loop");
        TV v[ND];
#pragma unroll
        for (int d = 0; d < ND; d++) v[d] = __ldg(base + d * 32);
#pragma unroll
        for (int d = 0; d < ND; d++) {
            const long j = i + off.o[d];
            if (j >= 0 && j < n) s += (Acc)v[d] * (Acc)__ldg(x + j);
        }
#endif
    } else {
        static_assert(!CC, "constant coefficients need a compiled diagonal count");
#pragma unroll 4
        for (int d = 0; d < off.nd; d++) {
            const long j = i + off.o[d];
            if (j >= 0 && j < n) {
                TX xj = __ldg(x + j);
                if constexpr (SC) xj = (TX)(xj * __ldg(xs + j));
                s += (Acc)__ldg(base + d * 32) * (Acc)xj;
            }
        }
    }
    return s;
}

template <int ND, typename TV, typename TX, typename Acc, class Epi, bool CC = false>
__global__ void __launch_bounds__(256, RB_DIA_MINB_ROWS)
k_sdia_rows(long n, DiaOff off, const TV* __restrict__ sv, const TX* __restrict__ x, Epi epi) {
    constexpr bool SC = ScaledGather<Epi>::value;
    const TX* xs = gather_scale_of<Epi, TX>(epi);
    const int lane = threadIdx.x & 31;
    const int nd = ND > 0 ? ND : off.nd;
    const long nslices = (n + 31) >> 5;
    double red = 0.0;
    for (long sl = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; sl < nslices;
         sl += ((long)gridDim.x * blockDim.x) >> 5) {
        const long i = (sl << 5) + lane;
#if RB_DIA_EPI_PREFETCH
        if constexpr (HasPre<Epi>::value) {
            // the epilogue's operands are loaded with the row's values and x
            typename Epi::Pre pr{};
            if (i < n) pr = epi.pre(i);
            const Acc s = sdia_row<ND, TV, TX, Acc, SC, CC>(i, n, off, sv + sl * nd * 32 + lane, x, xs);
            if (i < n) epi.post(i, s, red, pr);
        } else
#endif
        {
            const Acc s = sdia_row<ND, TV, TX, Acc, SC, CC>(i, n, off, sv + sl * nd * 32 + lane, x, xs);
            if (i < n) epi(i, s, red);
        }
    }
}

// (constant coefficients: 3 resident blocks, so that the 27 gathered FP64
// values of a row fit the register budget without spilling)
template <int ND, typename TV, class Fin, bool CC = false>
__global__ void __launch_bounds__(256, CC ? 3 : RB_DIA_MINB)
k_sdia_rows_dot(long n, DiaOff off, const TV* __restrict__ sv, const double* __restrict__ x,
                EpiStoreDot epi, ReduceSlot rs, Fin fin) {
    const int lane = threadIdx.x & 31;
    const int nd = ND > 0 ? ND : off.nd;
    const long nslices = (n + 31) >> 5;
    double red = 0.0;
    for (long sl = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; sl < nslices;
         sl += ((long)gridDim.x * blockDim.x) >> 5) {
        const long i = (sl << 5) + lane;
        const double s = sdia_row<ND, TV, double, double, false, CC>(i, n, off, sv + sl * nd * 32 + lane, x);
        if (i < n) epi(i, s, red);
    }
    block_reduce_finish(red, rs, fin);
}

inline unsigned dia_grid(long n, bool dot) {
    long blocks = ((n + 31) / 32 + 7) / 8;
    static const int per_sm_rows = grid_per_sm("RAPTOR_B200_GRID_DIA", RB_DIA_GRID_ROWS);
    static const int per_sm_dot = grid_per_sm("RAPTOR_B200_GRID_DIA_DOT", RB_DIA_GRID_DOT);
    long cap = (long)sm_count() * (dot ? per_sm_dot : per_sm_rows);
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (unsigned)blocks;
}

template <typename TV, typename TX, class Epi>
void launch_dia(const DiaOff& off, const TV* sv, long n, const TX* x, Epi epi) {
    if (n <= 0) return;
    using Acc = AccOf2<TV, TX>;
    if (off.mask && off.grid) {
        launch_grid<TX, Acc, Epi, false>(off, x, epi, NoFinish{});
        return;
    }
    const unsigned g = dia_grid(n, false);
    if (off.mask) {
        switch (off.nd) {
            case 5: k_sdia_rows<5, TV, TX, Acc, Epi, true><<<g, 256, 0, stream()>>>(n, off, sv, x, epi); break;
            case 7: k_sdia_rows<7, TV, TX, Acc, Epi, true><<<g, 256, 0, stream()>>>(n, off, sv, x, epi); break;
            case 9: k_sdia_rows<9, TV, TX, Acc, Epi, true><<<g, 256, 0, stream()>>>(n, off, sv, x, epi); break;
            default: k_sdia_rows<27, TV, TX, Acc, Epi, true><<<g, 256, 0, stream()>>>(n, off, sv, x, epi); break;
        }
        RB_CHECK_LAUNCH();
        return;
    }
    switch (off.nd) {
        case 5: k_sdia_rows<5, TV, TX, Acc, Epi><<<g, 256, 0, stream()>>>(n, off, sv, x, epi); break;
        case 7: k_sdia_rows<7, TV, TX, Acc, Epi><<<g, 256, 0, stream()>>>(n, off, sv, x, epi); break;
        case 9: k_sdia_rows<9, TV, TX, Acc, Epi><<<g, 256, 0, stream()>>>(n, off, sv, x, epi); break;
        case 27: k_sdia_rows<27, TV, TX, Acc, Epi><<<g, 256, 0, stream()>>>(n, off, sv, x, epi); break;
        default: k_sdia_rows<0, TV, TX, Acc, Epi><<<g, 256, 0, stream()>>>(n, off, sv, x, epi); break;
    }
    RB_CHECK_LAUNCH();
}

template <typename TV, class Fin>
void launch_dia_dot(const DiaOff& off, const TV* sv, long n, const double* x, double* y, Fin fin) {
    EpiStoreDot epi{x, y};
    if (off.mask && off.grid) {
        launch_grid<double, double, EpiStoreDot, true>(off, x, epi, fin);
        return;
    }
    const unsigned g = dia_grid(n, true);
    ReduceSlot rs = global_reduce_slot(g);
    if (off.mask) {
        switch (off.nd) {
            case 5: k_sdia_rows_dot<5, TV, Fin, true><<<g, 256, 0, stream()>>>(n, off, sv, x, epi, rs, fin); break;
            case 7: k_sdia_rows_dot<7, TV, Fin, true><<<g, 256, 0, stream()>>>(n, off, sv, x, epi, rs, fin); break;
            case 9: k_sdia_rows_dot<9, TV, Fin, true><<<g, 256, 0, stream()>>>(n, off, sv, x, epi, rs, fin); break;
            default: k_sdia_rows_dot<27, TV, Fin, true><<<g, 256, 0, stream()>>>(n, off, sv, x, epi, rs, fin); break;
        }
        RB_CHECK_LAUNCH();
        return;
    }
    switch (off.nd) {
        case 5: k_sdia_rows_dot<5, TV><<<g, 256, 0, stream()>>>(n, off, sv, x, epi, rs, fin); break;
        case 7: k_sdia_rows_dot<7, TV><<<g, 256, 0, stream()>>>(n, off, sv, x, epi, rs, fin); break;
        case 9: k_sdia_rows_dot<9, TV><<<g, 256, 0, stream()>>>(n, off, sv, x, epi, rs, fin); break;
        case 27: k_sdia_rows_dot<27, TV><<<g, 256, 0, stream()>>>(n, off, sv, x, epi, rs, fin); break;
        default: k_sdia_rows_dot<0, TV><<<g, 256, 0, stream()>>>(n, off, sv, x, epi, rs, fin); break;
    }
    RB_CHECK_LAUNCH();
}

// Whether every nonzero stored on diagonal d has one value: lo/hi[d] end as
// the least and greatest bit pattern (as FP64) of its nonzeros.  A block
// reduces its rows first (one atomic a diagonal a block: 7M rows' atomics
// on 27 addresses took 0.115 s at 192^3); launch with a grid of a few
// blocks a SM.
template <typename T>
__global__ void __launch_bounds__(256)
k_dia_const_range(long n, int nd, const T* __restrict__ dv, unsigned long long* lo,
                  unsigned long long* hi) {
    __shared__ unsigned long long smn[8], smx[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long nth = (long)gridDim.x * blockDim.x;
    for (int d = 0; d < nd; d++) {
        unsigned long long mn = ~0ull, mx = 0ull;
        for (long i = tid; i < n; i += nth) {
            const T v = dv[(i >> 5) * nd * 32 + d * 32 + (i & 31)];
            if (v != T(0)) {
                const unsigned long long b = (unsigned long long)__double_as_longlong((double)v);
                mn = b < mn ? b : mn;
                mx = b > mx ? b : mx;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long a = __shfl_xor_sync(0xffffffffu, mn, o);
            const unsigned long long c = __shfl_xor_sync(0xffffffffu, mx, o);
            mn = a < mn ? a : mn;
            mx = c > mx ? c : mx;
        }
        if (lane == 0) { smn[warp] = mn; smx[warp] = mx; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
                mn = smn[w] < mn ? smn[w] : mn;
                mx = smx[w] > mx ? smx[w] : mx;
            }
            if (mn != ~0ull) atomicMin(lo + d, mn);
            if (mx != 0ull) atomicMax(hi + d, mx);
        }
        __syncthreads();
    }
}

// bit d of mask[i]: a(i, i + o[d]) is nonzero
template <typename T>
__global__ void k_dia_mask(long n, int nd, const T* __restrict__ dv, unsigned* __restrict__ mask) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T* base = dv + (i >> 5) * nd * 32 + (i & 31);
    unsigned m = 0u;
    for (int d = 0; d < nd; d++)
        if (base[d * 32] != T(0)) m |= 1u << d;
    mask[i] = m;
}

// Sliced storage size (entries) for n rows and nd diagonals.
inline size_t sdia_size(long n, int nd) { return (size_t)((n + 31) / 32) * nd * 32; }

}  // namespace rb
