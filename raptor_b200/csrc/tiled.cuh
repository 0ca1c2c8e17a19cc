// tiled.cuh -- CSR row products with the gathered vector staged in shared
// memory, for the coarse operators of the cycle.
//
// A coarse Galerkin operator couples each row to rows a bounded distance
// away (for the 27-point hierarchy, two coarse planes either side), so a
// contiguous chunk of rows reads x only inside one window [lo, hi).  Here
// each block (one of kTileBlock threads per SM) takes a chunk, copies x's
// window into shared memory with coalesced loads, and then runs the usual
// row loop (G lanes a row, batches of index/value loads, the same
// summation order and shuffle tree as k_csr_rows) with every gather served
// by shared memory instead of L2.  The strided kernels are bound by the
// latency of those gathers; here only the value and index streams come from
// memory.  Used where the window of every chunk fits the shared memory a
// block may take and the timed product beats the other schedules (the lanes
// value then carries kRowsTiled).
#pragma once

#include "spmv.cuh"

namespace rb {

constexpr int kTileBlock = 1024;
// nonzeros a lane loads per batch (its gathers come from shared memory, so
// the batch only has to keep enough of the value and index streams in
// flight), and window entries a thread stages per round trip
constexpr int kTileBatch = 8;
constexpr int kTileStage = 8;
constexpr int kRowsTiled = 128;
// shared memory a block may hold (the B200 opt-in maximum is 227 KB)
constexpr int kTileSmemBytes = 220 * 1024;

// Chunk c = rows [c R, min(n, (c + 1) R)); lo[c] / hi[c] bound the columns
// its rows read (lo = hi = 0 for a chunk without entries).
static __global__ void k_row_windows(long n, int R, const int* __restrict__ rp,
                              const int* __restrict__ cols, const int* __restrict__ rbase,
                              const unsigned short* __restrict__ c16, int* lo, int* hi) {
    const int c = blockIdx.x;
    const long r0 = (long)c * R;
    const long r1 = r0 + R < n ? r0 + R : n;
    int mn = INT_MAX, mx = -1;
    for (long i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        const int b = rbase ? rbase[i] : 0;
        for (int j = rp[i]; j < rp[i + 1]; j++) {
            const int col = rbase ? b + (int)c16[j] : cols[j];
            mn = col < mn ? col : mn;
            mx = col > mx ? col : mx;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    __shared__ int smn[32], smx[32];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { smn[w] = mn; smx[w] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
            mn = min(mn, smn[k]);
            mx = max(mx, smx[k]);
        }
        lo[c] = mx >= 0 ? mn : 0;
        hi[c] = mx >= 0 ? mx + 1 : 0;
    }
}

// One chunk a block per loop step; I16 selects 16-bit column offsets
// (column = rbase[row] + c16[j]) over 32-bit columns.  A lane's nonzeros
// are summed in increasing position whatever the batch size, as in
// k_csr_rows.
template <int G, typename TV, typename TX, class Epi, bool I16>
__global__ void __launch_bounds__(kTileBlock, 1)
k_csr_rows_tiled(long n, const int* __restrict__ rp, const int* __restrict__ ci,
                 const int* __restrict__ rbase, const unsigned short* __restrict__ c16,
                 const TV* __restrict__ cv, const TX* __restrict__ x,
                 const int* __restrict__ wlo, const int* __restrict__ whi, int R, int nchunks,
                 Epi epi) {
    using Acc = AccOf2<TV, TX>;
    constexpr bool SC = ScaledGather<Epi>::value;
    constexpr int UN = kTileBatch;
    if constexpr (HasGate<Epi>::value) {
        if (!epi.open()) return;
    }
    extern __shared__ __align__(16) unsigned char tile_smem[];
    TX* xs = reinterpret_cast<TX*>(tile_smem);
    const TX* xsc = gather_scale_of<Epi, TX>(epi);
    constexpr int RPW = 32 / G;
    const int lane = threadIdx.x & 31;
    const int sub = lane / G, gl = lane & (G - 1);
    const int warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    double red = 0.0;
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const int w0 = wlo[c], len = whi[c] - wlo[c];
        // the window, kTileStage entries a thread in flight at a time
        for (int t0 = threadIdx.x; t0 < len; t0 += kTileStage * blockDim.x) {
            TX v[kTileStage];
#pragma unroll
            for (int u = 0; u < kTileStage; u++) {
                const int t = t0 + u * blockDim.x;
                v[u] = t < len ? __ldg(x + w0 + t) : TX(0);
                if constexpr (SC) v[u] = t < len ? (TX)(v[u] * __ldg(xsc + w0 + t)) : TX(0);
            }
#pragma unroll
            for (int u = 0; u < kTileStage; u++) {
                const int t = t0 + u * blockDim.x;
                if (t < len) xs[t] = v[u];
            }
        }
        __syncthreads();
        const long first = (long)c * R;
        const long last = first + R < n ? first + R : n;
        for (long base = first + (long)warp * RPW; base < last; base += (long)nw * RPW) {
            const long row = base + sub;
            const bool valid = row < last;
            int s = 0, e = 0, off = -w0;
            if (valid) {
                s = __ldg(rp + row);
                e = __ldg(rp + row + 1);
                if constexpr (I16) off += __ldg(rbase + row);
            }
            Acc sum = 0;
            for (int j = s + gl; j < e; j += UN * G) {
                int cc[UN];
                TV vv[UN];
#pragma unroll
                for (int q = 0; q < UN; q++) {
                    const bool ok = j + q * G < e;
                    if constexpr (I16) cc[q] = ok ? (int)__ldg(c16 + j + q * G) : 0;
                    else cc[q] = ok ? __ldg(ci + j + q * G) : 0;
                    vv[q] = ok ? __ldg(cv + j + q * G) : TV(0);
                }
                TX xx[UN];
#pragma unroll
                for (int q = 0; q < UN; q++) xx[q] = (j + q * G < e) ? xs[cc[q] + off] : TX(0);
#pragma unroll
                for (int q = 0; q < UN; q++)
                    if (j + q * G < e) sum += (Acc)vv[q] * (Acc)xx[q];
            }
            sum = group_sum<G>(sum);
            if (valid && gl == 0) epi(row, sum, red);
        }
        __syncthreads();
    }
    (void)red;
}

template <int G, typename TV, typename TX, class Epi, bool I16>
void launch_tiled_g(long n, const int* rp, const int* ci, const int* rbase,
                    const unsigned short* c16, const TV* cv, const TX* x, const int* lo,
                    const int* hi, int R, int nchunks, int wmax, Epi epi) {
    auto k = k_csr_rows_tiled<G, TV, TX, Epi, I16>;
    static bool attr = false;   // once per instantiation
    if (!attr) {
        RB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kTileSmemBytes));
        attr = true;
    }
    const int grid = nchunks < sm_count() ? nchunks : sm_count();
    k<<<grid, kTileBlock, (size_t)wmax * sizeof(TX), stream()>>>(n, rp, ci, rbase, c16, cv, x,
                                                                 lo, hi, R, nchunks, epi);
    RB_CHECK_LAUNCH();
}

template <typename TV, typename TX, class Epi, bool I16>
void launch_tiled(long n, const int* rp, const int* ci, const int* rbase,
                  const unsigned short* c16, const TV* cv, const TX* x, const int* lo,
                  const int* hi, int R, int nchunks, int wmax, Epi epi, int G) {
    if (n <= 0) return;
    switch (G) {
        case 1: launch_tiled_g<1, TV, TX, Epi, I16>(n, rp, ci, rbase, c16, cv, x, lo, hi, R, nchunks, wmax, epi); break;
        case 2: launch_tiled_g<2, TV, TX, Epi, I16>(n, rp, ci, rbase, c16, cv, x, lo, hi, R, nchunks, wmax, epi); break;
        case 4: launch_tiled_g<4, TV, TX, Epi, I16>(n, rp, ci, rbase, c16, cv, x, lo, hi, R, nchunks, wmax, epi); break;
        case 8: launch_tiled_g<8, TV, TX, Epi, I16>(n, rp, ci, rbase, c16, cv, x, lo, hi, R, nchunks, wmax, epi); break;
        case 16: launch_tiled_g<16, TV, TX, Epi, I16>(n, rp, ci, rbase, c16, cv, x, lo, hi, R, nchunks, wmax, epi); break;
        default: launch_tiled_g<32, TV, TX, Epi, I16>(n, rp, ci, rbase, c16, cv, x, lo, hi, R, nchunks, wmax, epi); break;
    }
}

}  // namespace rb
