// grid.cuh -- the box-grid form of a constant-coefficient stencil operator.
//
// A stencil_grid operator on an nx x ny x nz box (gallery/par_stencil.hpp) in
// the constant-coefficient form (DiaOff::mask, dia.cuh) has one value c_d per
// diagonal, and bit d of a row's mask is set exactly when the row's neighbour
// (z + dz_d, y + dy_d, x + dx_d) lies inside the box.  A clear bit adds
// c_d * 0 to the row's sum.  Here x is staged in shared memory one z-plane
// tile at a time, with a halo that reads 0 outside the box, and every row
// sums c_d * x(neighbour d) over all d in diagonal order, as the masked
// kernel does: the same products in the same order, so the results are
// equal bit for bit.  What changes is the work per row: the masked kernel
// forms 64-bit addresses, tests mask bits and issues a predicated global
// load per diagonal (bound by instruction issue, about 0.1 ms a sweep at
// 192^3), where this kernel reads each neighbour from shared memory at an
// offset the compiler knows (the stencil shape and tile are template
// parameters), and each plane tile is loaded from global memory once.
//
// Schedule: one block owns an x-y tile of TXW x TYH rows (VX adjacent rows
// in x a thread) and marches zc planes in z.  Four plane buffers form a
// ring: while the block computes output plane z from planes z-1, z, z+1, it
// loads plane z+2 into registers and stores it into the fourth buffer after
// its products, then one barrier.  The z loop is unrolled by four so every
// buffer index is a constant.
//
// Which operators take this form is decided at setup (find_grid, verified
// row by row on the device by k_grid_mask_check); 2D shapes run with the
// grid's y as the marching axis (ny = 1, tiles of 256 x 1).
//
// Included by dia.cuh after DiaOff and dia_coef.
#pragma once

#include "spmv.cuh"

namespace rb {

enum GridShape { kGridNone = 0, kBox27 = 1, kStar7 = 2, kBox9 = 3, kStar5 = 4 };

// (dz, dy, dx) of diagonal d of each shape, in ascending offset order (for
// nx >= 3 and, in 3D, ny >= 3, lexicographic (dz, dy, dx) order is the order
// of dz nx ny + dy nx + dx).  The 2D shapes are written on (z, x) with dy = 0.
template <int S> struct Shape;
template <> struct Shape<kBox27> {
    static constexpr int nd = 27, hy = 1;
    __host__ __device__ static constexpr int dz(int d) { return d / 9 - 1; }
    __host__ __device__ static constexpr int dy(int d) { return (d / 3) % 3 - 1; }
    __host__ __device__ static constexpr int dx(int d) { return d % 3 - 1; }
};
template <> struct Shape<kStar7> {
    static constexpr int nd = 7, hy = 1;
    __host__ __device__ static constexpr int dz(int d) { return d == 0 ? -1 : d == 6 ? 1 : 0; }
    __host__ __device__ static constexpr int dy(int d) { return d == 1 ? -1 : d == 5 ? 1 : 0; }
    __host__ __device__ static constexpr int dx(int d) { return d == 2 ? -1 : d == 4 ? 1 : 0; }
};
template <> struct Shape<kBox9> {
    static constexpr int nd = 9, hy = 0;
    __host__ __device__ static constexpr int dz(int d) { return d / 3 - 1; }
    __host__ __device__ static constexpr int dy(int) { return 0; }
    __host__ __device__ static constexpr int dx(int d) { return d % 3 - 1; }
};
template <> struct Shape<kStar5> {
    static constexpr int nd = 5, hy = 0;
    __host__ __device__ static constexpr int dz(int d) { return d == 0 ? -1 : d == 4 ? 1 : 0; }
    __host__ __device__ static constexpr int dy(int) { return 0; }
    __host__ __device__ static constexpr int dx(int d) { return d == 1 ? -1 : d == 3 ? 1 : 0; }
};

// Tile of a shape with VX adjacent rows in x a thread: TXW x TYH rows on
// NT threads, plane buffers of H rows of W values (W even, so that a pair of
// values at an even column is 2 TX aligned).
template <int S, int VX>
struct GridTile {
    static constexpr bool is3d = Shape<S>::hy == 1;
    static constexpr int TXT = is3d ? 32 : 256;   // threads along x
    static constexpr int TXW = TXT * VX, TYH = is3d ? 8 : 1;
    static constexpr int HY = Shape<S>::hy;
    static constexpr int W = TXW + 2, H = TYH + 2 * HY, P = W * H;
    static constexpr int NT = TXT * TYH;
    static constexpr int LPT = (P + NT - 1) / NT;   // plane values a thread loads
};

// The epilogue's operand record (an empty one when it has none).
struct NoPre {};
template <class Epi, class = void>
struct PreOf { using type = NoPre; };
template <class Epi>
struct PreOf<Epi, std::void_t<typename Epi::Pre>> { using type = typename Epi::Pre; };

// Resident blocks the compiler must allow for: the FP32 sweeps with two rows
// a thread (two or three operands a row: old iterate, b, inverse diagonal;
// the first sweep fused with the residual reads b and the inverse diagonal)
// are held to RB_GRID_MINB2 blocks of 256 threads (48 registers, no spills;
// the compiler's own choice is 64 registers, 4 blocks); the FP32 residual
// spills at 48 and keeps the compiler's choice.
#ifndef RB_GRID_MINB2
#define RB_GRID_MINB2 5
#endif
// The FP64 instances with two rows a thread and at most one operand a row
// (the outer A p with its dot, the FP64 residual) are held to
// RB_GRID_MINB_F64 blocks (64 registers, no spills; the compiler's choice
// for the dot is 78, 3 blocks); the FP64 sweeps spill at 64 and keep theirs.
#ifndef RB_GRID_MINB_F64
#define RB_GRID_MINB_F64 4
#endif
template <int VX, typename TX, class Epi>
constexpr int grid_min_blocks() {
    using Pre = typename PreOf<Epi>::type;
    if (VX == 2 && sizeof(TX) == 4 && sizeof(Pre) >= 2 * sizeof(TX)) return RB_GRID_MINB2;
    if (VX == 2 && sizeof(TX) == 8 && sizeof(Pre) <= sizeof(TX)) return RB_GRID_MINB_F64;
    return 0;
}

template <typename T> struct Pair;
template <> struct Pair<float> { using type = float2; };
template <> struct Pair<double> { using type = double2; };

// The in-box bits of row i's diagonals (x fastest).
template <int S>
__host__ __device__ inline unsigned grid_in_box_bits(long i, int nx, int ny, int nz) {
    const int xx = (int)(i % nx);
    const long t = i / nx;
    const int yy = (int)(t % ny), zz = (int)(t / ny);
    unsigned m = 0u;
    for (int d = 0; d < Shape<S>::nd; d++) {
        const int a = xx + Shape<S>::dx(d), b = yy + Shape<S>::dy(d), c = zz + Shape<S>::dz(d);
        if (a >= 0 && a < nx && b >= 0 && b < ny && c >= 0 && c < nz) m |= 1u << d;
    }
    return m;
}

// *bad = 1 when some row's mask is not the in-box bits of its coordinates.
template <int S>
__global__ void k_grid_mask_check(long n, int nx, int ny, int nz, const unsigned* __restrict__ mask,
                                  int* bad) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        if (mask[i] != grid_in_box_bits<S>(i, nx, ny, nz)) *bad = 1;
}

template <typename Acc>
__device__ __forceinline__ Acc fma_acc(Acc a, Acc b, Acc c);
template <>
__device__ __forceinline__ float fma_acc<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <>
__device__ __forceinline__ double fma_acc<double>(double a, double b, double c) { return __fma_rn(a, b, c); }

// y-epilogue of A x on the box grid (DOT: the epilogue accumulates a dot,
// reduced over the grid into fin).  One block per (x tile, y tile, z chunk),
// flattened into blockIdx.x with x fastest.  VX = 2: a thread computes rows
// x and x + 1 and reads, for each (plane, dy) its diagonals touch, the four
// values at x - 1 .. x + 2 as two aligned pairs; each row's products and
// their order are still those of VX = 1.
template <int S, int VX, typename TX, typename Acc, class Epi, bool DOT, class Fin>
__global__ void __launch_bounds__(GridTile<S, VX>::NT, grid_min_blocks<VX, TX, Epi>())
k_grid_rows(DiaOff off, const TX* __restrict__ x, Epi epi, ReduceSlot rs, Fin fin) {
    using G = GridTile<S, VX>;
    using Sh = Shape<S>;
    using TX2 = typename Pair<TX>::type;
    constexpr bool SC = ScaledGather<Epi>::value;
    __shared__ __align__(16) TX buf[4][G::P];
    if constexpr (!DOT && HasGate<Epi>::value) {
        if (!epi.open()) return;
    }
    const TX* xs = gather_scale_of<Epi, TX>(epi);
    const int nx = off.nx, ny = off.ny, nz = off.nz, zc = off.gzc;
    const int ntx = (nx + G::TXW - 1) / G::TXW, nty = (ny + G::TYH - 1) / G::TYH;
    const int bx = (int)(blockIdx.x % (unsigned)ntx);
    const int bt = (int)(blockIdx.x / (unsigned)ntx);
    const int by = bt % nty, bz = bt / nty;
    const int x0 = bx * G::TXW, y0 = by * G::TYH, z0 = bz * zc;
    const int tx = threadIdx.x % G::TXT, ty = threadIdx.x / G::TXT;
    const long plane = (long)nx * ny;

    // this thread's share of a plane tile: in-plane offset and whether it is
    // inside the box in x and y (the same for every plane)
    long goff[G::LPT];
    bool gok[G::LPT];
#pragma unroll
    for (int u = 0; u < G::LPT; u++) {
        const int e = threadIdx.x + u * G::NT;
        const int ry = e / G::W, rx = e % G::W;
        const int gy = y0 - G::HY + ry, gx = x0 - 1 + rx;
        gok[u] = e < G::P && gy >= 0 && gy < ny && gx >= 0 && gx < nx;
        goff[u] = (long)gy * nx + gx;
    }
    auto load = [&](int zp, TX (&v)[G::LPT]) {
        const bool zin = zp >= 0 && zp < nz;
        const long zb = (long)zp * plane;
#pragma unroll
        for (int u = 0; u < G::LPT; u++) {
            v[u] = TX(0);
            if (zin && gok[u]) {
                if constexpr (SC) v[u] = (TX)(__ldg(x + zb + goff[u]) * __ldg(xs + zb + goff[u]));
                else v[u] = __ldg(x + zb + goff[u]);
            }
        }
    };
    auto store = [&](int slot, const TX (&v)[G::LPT]) {
#pragma unroll
        for (int u = 0; u < G::LPT; u++) {
            const int e = threadIdx.x + u * G::NT;
            if (u < G::LPT - 1 || e < G::P) buf[slot][e] = v[u];
        }
    };
    const int zend = min(z0 + zc, nz);
    // buffer index of the value left of this thread's first row
    const int left = (ty + G::HY) * G::W + tx * VX;
    const int xr = x0 + tx * VX;
    const bool in_y = y0 + ty < ny;
    bool in_r[VX];
#pragma unroll
    for (int r = 0; r < VX; r++) in_r[r] = in_y && xr + r < nx;
    const long row_xy = (long)(y0 + ty) * nx + xr;
    {
        TX w[3][G::LPT];
        load(z0 - 1, w[0]);
        load(z0, w[1]);
        load(z0 + 1, w[2]);
        store(0, w[0]);
        store(1, w[1]);
        store(2, w[2]);
    }
    __syncthreads();

    double red = 0.0;
    // step K (output plane z): reads the buffers (K, K+1, K+2) mod 4 and
    // stores plane z + 2 (loaded at the step's start) into buffer (K + 3) mod
    // 4 when step z + 1 will need it
    auto step = [&](auto kc, int z) {
        constexpr int K = decltype(kc)::value;
        TX v[G::LPT];
        const bool more = z + 1 < zend;
        if (more) load(z + 2, v);
        const long i = (long)z * plane + row_xy;
        using Pre = typename PreOf<Epi>::type;
        Pre pr[VX] = {};
        if constexpr (HasPre<Epi>::value) {
#pragma unroll
            for (int r = 0; r < VX; r++)
                if (in_r[r]) pr[r] = epi.pre(i + r);
        }
        Acc s[VX];
#pragma unroll
        for (int r = 0; r < VX; r++) s[r] = Acc(0);
#pragma unroll
        for (int d = 0; d < Sh::nd; d++) {
            const TX* row = &buf[(K + 1 + Sh::dz(d)) & 3][left + Sh::dy(d) * G::W];
            const Acc c = dia_coef<Acc>(off, d);
            if constexpr (VX == 1) {
                s[0] = fma_acc<Acc>(c, (Acc)row[1 + Sh::dx(d)], s[0]);
            } else {
                // values at x - 1, x, x + 1, x + 2 (the same loads for every
                // diagonal of one (plane, dy), which the compiler merges)
                const TX2 a = *reinterpret_cast<const TX2*>(row);
                const TX2 b = *reinterpret_cast<const TX2*>(row + 2);
                const TX v0 = Sh::dx(d) < 0 ? a.x : Sh::dx(d) == 0 ? a.y : b.x;
                const TX v1 = Sh::dx(d) < 0 ? a.y : Sh::dx(d) == 0 ? b.x : b.y;
                s[0] = fma_acc<Acc>(c, (Acc)v0, s[0]);
                s[1] = fma_acc<Acc>(c, (Acc)v1, s[1]);
            }
        }
#pragma unroll
        for (int r = 0; r < VX; r++) {
            if (in_r[r]) {
                if constexpr (HasPre<Epi>::value) epi.post(i + r, s[r], red, pr[r]);
                else epi(i + r, s[r], red);
            }
        }
        if (more) store((K + 3) & 3, v);
        __syncthreads();
    };
    for (int z = z0; z < zend; z += 4) {
        step(std::integral_constant<int, 0>{}, z);
        if (z + 1 < zend) step(std::integral_constant<int, 1>{}, z + 1);
        if (z + 2 < zend) step(std::integral_constant<int, 2>{}, z + 2);
        if (z + 3 < zend) step(std::integral_constant<int, 3>{}, z + 3);
    }
    if constexpr (DOT) block_reduce_finish(red, rs, fin);
}

// Blocks of a launch: x tiles x y tiles x z chunks.
inline long grid_blocks(const DiaOff& off, int txw, int tyh) {
    const long ntx = (off.nx + txw - 1) / txw, nty = (off.ny + tyh - 1) / tyh;
    const long nzc = (off.nz + off.gzc - 1) / off.gzc;
    return ntx * nty * nzc;
}

template <int S, int VX, typename TX, typename Acc, class Epi, bool DOT, class Fin>
void launch_grid_vx(const DiaOff& off, const TX* x, Epi epi, Fin fin) {
    using G = GridTile<S, VX>;
    const long nb = grid_blocks(off, G::TXW, G::TYH);
    ReduceSlot rs{nullptr, nullptr};
    if constexpr (DOT) rs = global_reduce_slot((int)nb);
    k_grid_rows<S, VX, TX, Acc, Epi, DOT, Fin><<<(unsigned)nb, G::NT, 0, stream()>>>(off, x, epi, rs, fin);
    RB_CHECK_LAUNCH();
}

template <int S, typename TX, typename Acc, class Epi, bool DOT, class Fin>
void launch_grid_shape(const DiaOff& off, const TX* x, Epi epi, Fin fin) {
    if (off.gvx == 2) launch_grid_vx<S, 2, TX, Acc, Epi, DOT, Fin>(off, x, epi, fin);
    else launch_grid_vx<S, 1, TX, Acc, Epi, DOT, Fin>(off, x, epi, fin);
}

template <typename TX, typename Acc, class Epi, bool DOT, class Fin>
void launch_grid(const DiaOff& off, const TX* x, Epi epi, Fin fin) {
    switch (off.grid) {
        case kBox27: launch_grid_shape<kBox27, TX, Acc, Epi, DOT, Fin>(off, x, epi, fin); break;
        case kStar7: launch_grid_shape<kStar7, TX, Acc, Epi, DOT, Fin>(off, x, epi, fin); break;
        case kBox9: launch_grid_shape<kBox9, TX, Acc, Epi, DOT, Fin>(off, x, epi, fin); break;
        case kStar5: launch_grid_shape<kStar5, TX, Acc, Epi, DOT, Fin>(off, x, epi, fin); break;
        default: RB_REQUIRE(false, "unknown grid shape");
    }
}

}  // namespace rb
