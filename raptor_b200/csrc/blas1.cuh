// blas1.cuh -- vector kernels of the V-cycle and the Krylov loops, the
// device-side Krylov scalars, and the coarse-level dense LU.
#pragma once

#include "spmv.cuh"

namespace rb {

// Iteration state of the PCG loop run on the device (RB_PCG_TRUE_RESIDUAL):
// the host writes it before each launch of the loop's graph, the last kernel
// of every iteration advances it.
constexpr int kPcgChunk = 16;   // iterations one launch of the loop graph may run
struct PcgCtl {
    int it;           // iterations done
    int chunk_base;   // first iteration of this launch
    int chunk_end;    // last iteration this launch may run
    int pmode;        // at the start of the next iteration: 0 keep p, 1 p = z + beta p
    double tol_bb;    // the stopping threshold tol * ||b||
};

// Krylov scalars live on the device so a whole iteration can be replayed
// from a CUDA graph without host round trips.
struct KScal {
    double rz;        // r.z of the current iterate
    double rz_prev;
    double pAp;
    double alpha;
    double beta;
    double rr;        // r.r (recurrence residual)
    double bb;        // b.b
    double tmp;
    int breakdown;    // p.Ap < 0 or not finite
    int pad;
    PcgCtl ctl;
    double chunk_rr[kPcgChunk];   // r.r after each iteration of the launch
};

template <typename TO, typename TI>
__global__ void k_convert(long n, const TI* __restrict__ in, TO* __restrict__ out) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (TO)in[i];
}

// x = dinv .* b (first Jacobi sweep from a zero guess: A*0 = 0)
template <typename TB, typename T>
__global__ void k_scale_first(long n, const TB* __restrict__ b, const T* __restrict__ dinv,
                              T* __restrict__ x) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = (T)((T)b[i] * dinv[i]);
}

// y = x + yp (prolongation into a second buffer is done by the row kernel)
template <typename T>
__global__ void k_fill(long n, T* __restrict__ x, T v) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = v;
}

template <typename T>
__global__ void k_axpy(long n, T* __restrict__ y, const T* __restrict__ x, double a) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i] * (T)a;
}

template <typename T>
__global__ void k_scale(long n, T* __restrict__ y, double a) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] *= (T)a;
}

// ------------------------------------------------- Krylov fused updates --
// x += alpha p ; r -= alpha Ap ; rr = r.r   (par_cg.cpp:206-217)
struct FinSetRR {
    KScal* s;
    __device__ void operator()(double t) const { s->rr = t; }
};

template <class Fin>
__global__ void __launch_bounds__(256)
k_cg_update(long n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
            const double* __restrict__ Ap, const KScal* __restrict__ s, int update_r,
            ReduceSlot rs, Fin fin) {
    const double alpha = s->alpha;
    double t = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        x[i] += p[i] * alpha;
        if (update_r) {
            double ri = r[i] + Ap[i] * (-1.0 * alpha);
            r[i] = ri;
            t += ri * ri;
        }
    }
    block_reduce_finish(t, rs, fin);
}

// p = z + beta p  (or p = z on a restart), par_cg.cpp:234-243
template <typename TZ>
static __global__ void k_cg_p(long n, double* __restrict__ p, const TZ* __restrict__ z,
                       const KScal* __restrict__ s, int restart) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (restart) p[i] = (double)z[i];
    else p[i] = p[i] * s->beta + (double)z[i];
}

// p = z + beta p at the start of an iteration of the device-side loop, or
// nothing when the previous step left p = z (start, restart)
template <typename TZ>
static __global__ void k_cg_p_dev(long n, double* __restrict__ p, const TZ* __restrict__ z,
                                  const KScal* __restrict__ s) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || s->ctl.pmode == 0) return;
    p[i] = p[i] * s->beta + (double)z[i];
}

// Last kernel of one iteration of the device-side loop: count the iteration,
// keep its r.r for the host's residual history, ask for the p update next
// time, and (use_cond) end the graph's while loop once the iteration broke
// down, met the tolerance (the host then confirms it with b - A x) or
// reached the last iteration of this launch.
static __global__ void k_pcg_step_end(KScal* s, cudaGraphConditionalHandle h, int use_cond) {
    if (threadIdx.x != 0) return;
    const int it = s->ctl.it + 1;
    s->ctl.it = it;
    const int slot = it - s->ctl.chunk_base;
    if (slot >= 0 && slot < kPcgChunk) s->chunk_rr[slot] = s->rr;
    s->ctl.pmode = 1;
    if (use_cond) {
        const bool stop = s->breakdown != 0 || sqrt(s->rr) <= s->ctl.tol_bb || it >= s->ctl.chunk_end ||
                          slot + 1 >= kPcgChunk;
        cudaGraphSetConditional(h, stop ? 0u : 1u);
    }
}

// generic deterministic dot into a KScal field through a finisher
template <class Fin>
__global__ void __launch_bounds__(256)
k_dot_fin(const double* __restrict__ a, const double* __restrict__ b, long n, ReduceSlot rs,
          Fin fin) {
    double t = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        t += a[i] * b[i];
    block_reduce_finish(t, rs, fin);
}

// ----------------------------------------------------------- dense LU --
// Coarsest level: the reference gathers A_c row-major and hands it to
// column-major dgetrf_, which therefore factors A_c^T, then solves with
// dgetrs_('N') (multilevel/par_multilevel.hpp:295-331, 360-374).  One CTA,
// partial pivoting on the first largest |entry| like idamax.
static __global__ void k_dense_from_csr(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                 const double* __restrict__ cv, double* a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int j = rp[i]; j < rp[i + 1]; j++) a[(size_t)i * n + ci[j]] = cv[j];
}

static __global__ void k_lu_factor(int n, double* a, int* piv, int* info) {
    __shared__ double sval[1024];
    __shared__ int sidx[1024];
    __shared__ int p_s;
    for (int k = 0; k < n; k++) {
        // pivot search in column k, rows k..n-1 (first maximum)
        double best = -1.0;
        int bi = n;
        for (int i = k + threadIdx.x; i < n; i += blockDim.x) {
            double v = fabs(a[i + (size_t)k * n]);
            if (v > best) { best = v; bi = i; }
        }
        sval[threadIdx.x] = best;
        sidx[threadIdx.x] = bi;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) {
                double v2 = sval[threadIdx.x + s];
                int i2 = sidx[threadIdx.x + s];
                if (v2 > sval[threadIdx.x] || (v2 == sval[threadIdx.x] && i2 < sidx[threadIdx.x])) {
                    sval[threadIdx.x] = v2;
                    sidx[threadIdx.x] = i2;
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            p_s = sidx[0] < n ? sidx[0] : k;
            piv[k] = p_s;
            if (a[p_s + (size_t)k * n] == 0.0 && *info == 0) *info = k + 1;
        }
        __syncthreads();
        const int p = p_s;
        if (p != k)
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                double t = a[k + (size_t)j * n];
                a[k + (size_t)j * n] = a[p + (size_t)j * n];
                a[p + (size_t)j * n] = t;
            }
        __syncthreads();
        const double d = a[k + (size_t)k * n];
        if (d != 0.0)
            for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) a[i + (size_t)k * n] /= d;
        __syncthreads();
        for (int idx = threadIdx.x; idx < (n - k - 1) * (n - k - 1); idx += blockDim.x) {
            int i = k + 1 + idx % (n - k - 1);
            int j = k + 1 + idx / (n - k - 1);
            a[i + (size_t)j * n] -= a[i + (size_t)k * n] * a[k + (size_t)j * n];
        }
        __syncthreads();
    }
}

// Solve (LU) x = b for one right-hand side held in T; arithmetic in FP64.
template <typename T>
__global__ void k_lu_solve(int n, const double* __restrict__ lu, const int* __restrict__ piv,
                           const T* __restrict__ b, T* __restrict__ x) {
    extern __shared__ double y[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = (double)b[i];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < n; k++) {
            int p = piv[k];
            if (p != k) { double t = y[k]; y[k] = y[p]; y[p] = t; }
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
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = (T)y[i];
}

// Coarse levels of up to kCoarseInvMax rows are solved by one dense product
// with the inverse of the factored matrix (built once at setup from the LU,
// column by column): a coarse solve then needs one read of the inverse and
// no sequential substitution steps.
constexpr int kCoarseInvMax = 512;

// inv (column-major, n x n) = the inverse of the matrix factored in lu/piv.
static __global__ void k_lu_invert(int n, const double* __restrict__ lu, const int* __restrict__ piv,
                                   double* __restrict__ inv) {
    extern __shared__ double y[];
    for (int c = 0; c < n; c++) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = (i == c) ? 1.0 : 0.0;
        __syncthreads();
        if (threadIdx.x == 0)
            for (int k = 0; k < n; k++) {
                const int p = piv[k];
                if (p != k) { double t = y[k]; y[k] = y[p]; y[p] = t; }
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
        for (int i = threadIdx.x; i < n; i += blockDim.x) inv[(size_t)c * n + i] = y[i];
        __syncthreads();
    }
}

// x = inv b for column blockIdx.x of k interleaved columns (k = 1: a vector)
template <typename T>
__global__ void k_coarse_mv(int n, const double* __restrict__ inv, int k, const T* __restrict__ b,
                            T* __restrict__ x) {
    extern __shared__ double bs[];
    const int c = blockIdx.x;
    for (int i = threadIdx.x; i < n; i += blockDim.x) bs[i] = (double)b[(long)i * k + c];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < n; j++) s += inv[(size_t)j * n + i] * bs[j];
        x[(long)i * k + c] = (T)s;
    }
}

}  // namespace rb
