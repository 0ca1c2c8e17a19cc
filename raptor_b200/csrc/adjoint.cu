// adjoint.cu -- the differentiation form: finite-volume assembly of a
// variable-coefficient diffusion operator, its backward pass, the SDDMM
// that turns the adjoint and primal solutions into dL/dA, and the adjoint
// solve A^T lambda = dL/dx through the AMG hierarchy built for A.
//
// Operator: -div(k grad u) = b on an nx x ny grid of unit cells, cell
// c = y nx + x, homogeneous Dirichlet walls.  The face between neighbouring
// cells i, j has transmissibility t_ij = 2 k_i k_j / (k_i + k_j) (harmonic
// mean); a wall face of cell i has t = 2 k_i (half a cell to the wall).
// A_ii = sum of the cell's face transmissibilities, A_ij = -t_ij; rows
// list their columns in increasing order (i - nx, i - 1, i, i + 1, i + nx).
// The reference has no differentiation path; everything here is new.
#include <algorithm>
#include <cmath>
#include <memory>

#include "hierarchy.cuh"

namespace rb {

namespace {

__device__ __forceinline__ double harm(double a, double b) { return 2.0 * a * b / (a + b); }

__global__ void k_fv_count(int nx, int ny, int* cnt) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long)nx * ny) return;
    const int x = (int)(c % nx), y = (int)(c / nx);
    cnt[c] = 1 + (y > 0) + (x > 0) + (x < nx - 1) + (y < ny - 1);
}

__global__ void k_fv_fill(int nx, int ny, const double* __restrict__ k, const int* __restrict__ rp,
                          int* ci, double* cv) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long)nx * ny) return;
    const int x = (int)(c % nx), y = (int)(c / nx);
    const double kc = k[c];
    int j = rp[c];
    double diag = 0.0;
    // in increasing column order
    if (y > 0) {
        const double t = harm(kc, k[c - nx]);
        ci[j] = (int)(c - nx); cv[j++] = -t; diag += t;
    } else {
        diag += 2.0 * kc;
    }
    if (x > 0) {
        const double t = harm(kc, k[c - 1]);
        ci[j] = (int)(c - 1); cv[j++] = -t; diag += t;
    } else {
        diag += 2.0 * kc;
    }
    const int jd = j++;
    if (x < nx - 1) {
        const double t = harm(kc, k[c + 1]);
        ci[j] = (int)(c + 1); cv[j++] = -t; diag += t;
    } else {
        diag += 2.0 * kc;
    }
    if (y < ny - 1) {
        const double t = harm(kc, k[c + nx]);
        ci[j] = (int)(c + nx); cv[j++] = -t; diag += t;
    } else {
        diag += 2.0 * kc;
    }
    ci[jd] = (int)c;
    cv[jd] = diag;
}

__device__ __forceinline__ int find_col(const int* __restrict__ rp, const int* __restrict__ ci,
                                        long row, long col) {
    for (int j = rp[row]; j < rp[row + 1]; j++)
        if (ci[j] == col) return j;
    return -1;
}

// dL/dk_c from dL/dA (gA on A's pattern): each face f of cell c contributes
// dL/dt_f dt_f/dk_c, with dL/dt_f = gA_cc + gA_nn - gA_cn - gA_nc for an
// interior face and gA_cc for a wall face (dt/dk_c = 2 there).
__global__ void k_fv_backward(int nx, int ny, const double* __restrict__ k,
                              const int* __restrict__ rp, const int* __restrict__ ci,
                              const double* __restrict__ gA, double* __restrict__ gk, int* bad) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long)nx * ny) return;
    const int x = (int)(c % nx), y = (int)(c / nx);
    const double kc = k[c];
    const int jcc = find_col(rp, ci, c, c);
    if (jcc < 0) { atomicAdd(bad, 1); return; }
    const double gcc = gA[jcc];
    double g = 0.0;
    const long nb[4] = {c - nx, c - 1, c + 1, c + nx};
    const bool in[4] = {y > 0, x > 0, x < nx - 1, y < ny - 1};
#pragma unroll
    for (int f = 0; f < 4; f++) {
        if (!in[f]) {
            g += gcc * 2.0;
            continue;
        }
        const long n = nb[f];
        const int jcn = find_col(rp, ci, c, n), jnc = find_col(rp, ci, n, c);
        const int jnn = find_col(rp, ci, n, n);
        if (jcn < 0 || jnc < 0 || jnn < 0) { atomicAdd(bad, 1); return; }
        const double dLdt = gcc + gA[jnn] - gA[jcn] - gA[jnc];
        const double kn = k[n], s = kc + kn;
        g += dLdt * (2.0 * kn * kn / (s * s));
    }
    gk[c] = g;
}

// SDDMM on A's pattern: out_j = scale lambda_i x_{col(j)}
__global__ void k_sddmm(long n, const int* __restrict__ rp, const int* __restrict__ ci,
                        const double* __restrict__ lambda, const double* __restrict__ x,
                        double scale, double* __restrict__ out) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double li = lambda[i] * scale;
    for (int j = rp[i]; j < rp[i + 1]; j++) out[j] = li * x[ci[j]];
}

// |A_ij - A_ji| over the stored pattern (and a missing mirror counts):
// sets *asym when the matrix is not symmetric to within tol relative.
__global__ void k_symmetry(long n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ cv, double tol, int* asym) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int j = rp[i]; j < rp[i + 1]; j++) {
        const long c = ci[j];
        if (c == i) continue;
        double m = 0.0;
        bool found = false;
        for (int q = rp[c]; q < rp[c + 1]; q++)
            if (ci[q] == i) { m = cv[q]; found = true; break; }
        const double v = cv[j];
        if (!found ? v != 0.0 : fabs(v - m) > tol * fmax(fabs(v), fabs(m))) {
            atomicAdd(asym, 1);
            return;
        }
    }
}

}  // namespace

rb_csr_s* fv_assemble(int nx, int ny, const double* k_dev) {
    RB_REQUIRE(nx >= 1 && ny >= 1, "fv_assemble: empty grid");
    const long n = (long)nx * ny;
    RB_REQUIRE(n * 5 <= INT_MAX, "fv_assemble: grid too large for int32 indices");
    DevArray<int> cnt((size_t)n);
    k_fv_count<<<grid_for(n, 256), 256, 0, stream()>>>(nx, ny, cnt.get());
    RB_CHECK_LAUNCH();
    rb_csr_s* A = new_csr((int)n, (int)n, 0);
    const long long nnz = exclusive_scan(cnt.get(), A->rowptr.get(), (int)n);
    A->nnz = nnz;
    A->cols.alloc((size_t)nnz);
    A->vals.alloc((size_t)nnz);
    k_fv_fill<<<grid_for(n, 256), 256, 0, stream()>>>(nx, ny, k_dev, A->rowptr.get(), A->cols.get(),
                                                      A->vals.get());
    RB_CHECK_LAUNCH();
    return A;
}

void fv_backward(int nx, int ny, const double* k_dev, const rb_csr_s& A, const double* gA,
                 double* gk) {
    const long n = (long)nx * ny;
    RB_REQUIRE(A.n_rows == n && A.n_cols == n, "fv_backward: A does not match the grid");
    DevArray<int> bad(1);
    bad.zero();
    k_fv_backward<<<grid_for(n, 256), 256, 0, stream()>>>(nx, ny, k_dev, A.rowptr.get(),
                                                          A.cols.get(), gA, gk, bad.get());
    RB_CHECK_LAUNCH();
    RB_REQUIRE(read_scalar(bad.get()) == 0, "fv_backward: A lacks the 5-point pattern of the grid");
}

void sddmm(const rb_csr_s& A, const double* lambda, const double* x, double scale, double* out) {
    const long n = A.n_rows;
    if (n == 0) return;
    k_sddmm<<<grid_for(n, 256), 256, 0, stream()>>>(n, A.rowptr.get(), A.cols.get(), lambda, x,
                                                    scale, out);
    RB_CHECK_LAUNCH();
}

bool is_symmetric(const rb_csr_s& A, double tol) {
    if (A.n_rows != A.n_cols) return false;
    DevArray<int> asym(1);
    asym.zero();
    if (A.n_rows)
        k_symmetry<<<grid_for(A.n_rows, 256), 256, 0, stream()>>>(
            A.n_rows, A.rowptr.get(), A.cols.get(), A.vals.get(), tol, asym.get());
    RB_CHECK_LAUNCH();
    return read_scalar(asym.get()) == 0;
}

}  // namespace rb

namespace rb {

// The adjoint solve A^T lambda = g reuses the hierarchy of A.  The transpose
// of a V-cycle M is the V-cycle for A^T with restriction P^T, prolongation
// R^T, the transposed smoother (for Jacobi-type sweeps the same diagonal),
// pre- and post-smoothing swapped, and the transposed coarse solve.  With
// R = P^T stored, restriction and prolongation use the same R and P; with
// equal pre- and post-sweeps the order is unchanged.  So:
//   * A symmetric (checked once per operator): every A_l = R A_{l-1} P is
//     symmetric, M^T = M, and the adjoint is the same PCG;
//   * otherwise a second hierarchy holds the transposed cycle -- A_l^T on
//     every level, the same P and R, the forward smoother's diagonals, and
//     the coarse LU of A_c -- and right-preconditioned BiCGStab solves with
//     A^T (CG needs a symmetric operator).
int adjoint_solve(const rb_csr_s& A, Hierarchy& H, double* lambda, const double* g, double tol,
                  int max_iter, int* iters, double* relres) {
    const long n = A.n_rows;
    RB_REQUIRE(n == H.master[0].A->n_rows, "adjoint: A and the hierarchy differ in size");
    if (H.adj_A != &A) {
        H.adj_sym = is_symmetric(A, 1e-14);
        H.adj_A = &A;
        H.adj.reset();
        H.adj_AT.reset();
    }
    RB_CUDA(cudaMemsetAsync(lambda, 0, sizeof(double) * n, stream()));
    int rc, nh = 0;
    const long cap = (max_iter > 0 ? max_iter : (long)(1.3 * n) + 2) + 2;
    std::vector<double> hist((size_t)cap);
    if (H.adj_sym) {
        rc = H.pcg(A, lambda, g, tol, max_iter, RB_PCG_TRUE_RESIDUAL, hist.data(), (int)cap, &nh);
    } else {
        const int rt = H.opts.relax_type;
        RB_REQUIRE((rt == RB_RELAX_JACOBI && !H.opts.jacobi_compat) || rt == RB_RELAX_L1JACOBI,
                   "adjoint of a nonsymmetric operator: the smoother must be Jacobi or L1-Jacobi");
        if (!H.adj) {
            const int L = H.num_levels();
            std::unique_ptr<Hierarchy> T(new Hierarchy());
            T->opts = H.opts;
            T->use_graphs = H.use_graphs;
            T->master.resize(L);
            for (int l = 0; l < L; l++) {
                rb_csr_s* At = transpose(*H.master[l].A);
                sort_rows_diag_first(*At, true);
                T->master[l].A.reset(At);
                if (l < L - 1) {
                    T->master[l].P.reset(clone_csr(*H.master[l].P));
                    T->master[l].R.reset(clone_csr(*H.master[l].R));
                }
            }
            T->build_cycle_data();
            // the transposed smoother keeps the forward diagonals
            for (int l = 0; l < L - 1; l++) {
                if (H.opts.precision == RB_PREC_FP32)
                    RB_CUDA(cudaMemcpyAsync(T->lv32[l].dinv.get(), H.lv32[l].dinv.get(),
                                            sizeof(float) * T->lv32[l].n, cudaMemcpyDeviceToDevice,
                                            stream()));
                else
                    RB_CUDA(cudaMemcpyAsync(T->lv64[l].dinv.get(), H.lv64[l].dinv.get(),
                                            sizeof(double) * T->lv64[l].n, cudaMemcpyDeviceToDevice,
                                            stream()));
            }
            H.adj_AT.reset(transpose(A));
            T->src_A = H.adj_AT.get();
            H.adj = std::move(T);
        }
        rc = krylov_bicgstab(*H.adj_AT, H.adj.get(), lambda, g, tol, max_iter, hist.data(),
                             (int)cap, &nh);
    }
    // the true relative residual of the adjoint system
    const rb_csr_s& Aop = H.adj_sym ? A : *H.adj_AT;
    DevArray<double> r((size_t)n + 1);
    residual64(view(Aop), lambda, g, r.get());
    const double rn = H.norm64(r.get(), n), gn = H.norm64(g, n);
    if (iters) *iters = std::max(nh - 1, 0);
    if (relres) *relres = gn > 0 ? rn / gn : rn;
    return rc;
}

}  // namespace rb
