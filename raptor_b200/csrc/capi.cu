// capi.cu -- the extern "C" boundary (include/raptor_b200.h).
//
// Every entry point catches library errors and CUDA failures and turns them
// into an rb_status plus a per-thread message; nothing throws across the C
// boundary.  There is no host fallback: without a device every compute call
// fails with RB_ERR_NO_DEVICE.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "blas1.cuh"
#include "bsr.cuh"
#include "hierarchy.cuh"
#include "rb_internal.cuh"

namespace rb {
const char* last_error_cstr();
ReduceSlot global_reduce_slot(int grid);
}  // namespace rb

using namespace rb;

namespace {

template <class F>
int guarded(F&& f) {
    try {
        set_last_error("");
        return f();
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return RB_ERR_OOM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return RB_ERR_INVALID;
    }
}

bool g_init = false;

void ensure_device() {
    if (g_init) return;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) throw Error(RB_ERR_NO_DEVICE, "no CUDA device available");
    RB_CUDA(cudaSetDevice(0));
    (void)stream();
    g_init = true;
}

#define NEED(p) RB_REQUIRE((p) != nullptr, #p " is NULL")

}  // namespace

extern "C" {

const char* rb_last_error(void) { return last_error_cstr(); }

const char* rb_version(void) { return "raptor_b200 1.0 (sm_100a)"; }

int rb_init(int device) {
    return guarded([&]() -> int {
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0) throw Error(RB_ERR_NO_DEVICE, "no CUDA device available");
        RB_REQUIRE(device >= 0 && device < n, "device index out of range");
        RB_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        RB_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major != 10)
            throw Error(RB_ERR_NO_DEVICE, "libraptor_b200 holds sm_100a kernels only; device is sm_" +
                                              std::to_string(prop.major) + std::to_string(prop.minor));
        (void)stream();
        g_init = true;
        return RB_OK;
    });
}

int rb_set_stream(void* s) {
    return guarded([&]() -> int {
        ensure_device();
        set_stream((cudaStream_t)s);
        return RB_OK;
    });
}

int rb_synchronize(void) {
    return guarded([&]() -> int {
        ensure_device();
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

// ------------------------------------------------------------ containers --
int rb_csr_create(int n_rows, int n_cols, int64_t nnz, const int* rowptr, const int* cols,
                  const double* vals, int on_device, rb_csr* out) {
    return guarded([&]() -> int {
        ensure_device();
        NEED(out); NEED(rowptr);
        RB_REQUIRE(nnz == 0 || (cols && vals), "cols/vals are NULL");
        std::unique_ptr<rb_csr_s> A(new_csr(n_rows, n_cols, nnz));
        auto kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        if (!on_device) {
            RB_REQUIRE(rowptr[0] == 0 && rowptr[n_rows] == nnz, "rowptr does not span nnz");
            for (int i = 0; i < n_rows; i++)
                RB_REQUIRE(rowptr[i] <= rowptr[i + 1], "rowptr is not monotone");
            for (int64_t j = 0; j < nnz; j++)
                RB_REQUIRE(cols[j] >= 0 && cols[j] < n_cols, "column index out of range");
        }
        RB_CUDA(cudaMemcpyAsync(A->rowptr.get(), rowptr, sizeof(int) * ((size_t)n_rows + 1), kind, stream()));
        if (nnz) {
            RB_CUDA(cudaMemcpyAsync(A->cols.get(), cols, sizeof(int) * nnz, kind, stream()));
            RB_CUDA(cudaMemcpyAsync(A->vals.get(), vals, sizeof(double) * nnz, kind, stream()));
        }
        RB_CUDA(cudaStreamSynchronize(stream()));
        *out = A.release();
        return RB_OK;
    });
}

int rb_csr_destroy(rb_csr A) {
    return guarded([&]() -> int {
        delete A;
        return RB_OK;
    });
}

int rb_csr_info(rb_csr A, int* n_rows, int* n_cols, int64_t* nnz) {
    return guarded([&]() -> int {
        NEED(A);
        if (n_rows) *n_rows = A->n_rows;
        if (n_cols) *n_cols = A->n_cols;
        if (nnz) *nnz = A->nnz;
        return RB_OK;
    });
}

int rb_csr_download(rb_csr A, int* rowptr, int* cols, double* vals) {
    return guarded([&]() -> int {
        NEED(A);
        if (rowptr) A->rowptr.download(rowptr, (size_t)A->n_rows + 1);
        if (cols) A->cols.download(cols, (size_t)A->nnz);
        if (vals) A->vals.download(vals, (size_t)A->nnz);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_csr_device_arrays(rb_csr A, int** rowptr, int** cols, double** vals) {
    return guarded([&]() -> int {
        NEED(A);
        if (rowptr) *rowptr = A->rowptr.get();
        if (cols) *cols = A->cols.get();
        if (vals) *vals = A->vals.get();
        return RB_OK;
    });
}

int rb_csr_sort_diag_first(rb_csr A) {
    return guarded([&]() -> int {
        NEED(A);
        sort_rows_diag_first(*A, true);
        RB_CHECK_LAUNCH();
        A->tmap.reset();  // entry positions moved
        return RB_OK;
    });
}

int rb_csr_transpose(rb_csr A, rb_csr* out) {
    return guarded([&]() -> int {
        NEED(A); NEED(out);
        *out = transpose(*A);
        return RB_OK;
    });
}

// --------------------------------------------------------------- vectors --
int rb_vec_create(int n, rb_vec* out) {
    return guarded([&]() -> int {
        ensure_device();
        NEED(out);
        RB_REQUIRE(n >= 0, "negative vector size");
        auto* v = new rb_vec_s();
        v->n = n;
        v->v.alloc((size_t)n + 1);
        v->v.zero();
        *out = v;
        return RB_OK;
    });
}

int rb_vec_destroy(rb_vec v) {
    return guarded([&]() -> int {
        delete v;
        return RB_OK;
    });
}

int rb_vec_size(rb_vec v, int* n) {
    return guarded([&]() -> int {
        NEED(v); NEED(n);
        *n = v->n;
        return RB_OK;
    });
}

// host or device source/destination (unified addressing decides the copy)
int rb_vec_upload(rb_vec v, const double* host) {
    return guarded([&]() -> int {
        NEED(v); NEED(host);
        if (v->n)
            RB_CUDA(cudaMemcpyAsync(v->v.get(), host, sizeof(double) * v->n, cudaMemcpyDefault,
                                    stream()));
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_vec_download(rb_vec v, double* host) {
    return guarded([&]() -> int {
        NEED(v); NEED(host);
        if (v->n)
            RB_CUDA(cudaMemcpyAsync(host, v->v.get(), sizeof(double) * v->n, cudaMemcpyDefault,
                                    stream()));
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_vec_set(rb_vec v, double value) {
    return guarded([&]() -> int {
        NEED(v);
        if (v->n) k_fill<double><<<grid_for(v->n, 256), 256, 0, stream()>>>(v->n, v->v.get(), value);
        RB_CHECK_LAUNCH();
        return RB_OK;
    });
}

int rb_vec_device_ptr(rb_vec v, double** ptr) {
    return guarded([&]() -> int {
        NEED(v); NEED(ptr);
        *ptr = v->v.get();
        return RB_OK;
    });
}

int rb_vec_copy(rb_vec dst, rb_vec src) {
    return guarded([&]() -> int {
        NEED(dst); NEED(src);
        RB_REQUIRE(dst->n == src->n, "vector sizes differ");
        RB_CUDA(cudaMemcpyAsync(dst->v.get(), src->v.get(), sizeof(double) * dst->n,
                                cudaMemcpyDeviceToDevice, stream()));
        return RB_OK;
    });
}

int rb_vec_axpy(rb_vec y, rb_vec x, double a) {
    return guarded([&]() -> int {
        NEED(y); NEED(x);
        RB_REQUIRE(y->n == x->n, "vector sizes differ");
        if (y->n) k_axpy<double><<<grid_for(y->n, 256), 256, 0, stream()>>>(y->n, y->v.get(), x->v.get(), a);
        RB_CHECK_LAUNCH();
        return RB_OK;
    });
}

// out[k] = x[idx[k]]: packing the values a halo exchange sends.  An index
// outside x gives NaN instead of a read out of bounds.
__global__ void k_vec_gather(int n, const double* __restrict__ x, int nx, const int* __restrict__ idx,
                             double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int j = idx[k];
    out[k] = (j >= 0 && j < nx) ? x[j] : __longlong_as_double(0x7ff8000000000000ll);
}

int rb_vec_gather(rb_vec x, const int* idx, int n, double* out) {
    return guarded([&]() -> int {
        NEED(x);
        RB_REQUIRE(n >= 0, "negative count");
        RB_REQUIRE(n == 0 || (idx && out), "null index or output pointer");
        if (n) k_vec_gather<<<grid_for(n, 256), 256, 0, stream()>>>(n, x->v.get(), x->n, idx, out);
        RB_CHECK_LAUNCH();
        return RB_OK;
    });
}

// y[idx[k]] += v[k]: adding a transpose exchange's received values into the
// owner's rows.  The indices of one call must be distinct (one message);
// an index outside y is skipped.
__global__ void k_vec_scatter_add(int n, double* __restrict__ y, int ny, const int* __restrict__ idx,
                                  const double* __restrict__ v) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int j = idx[k];
    if (j >= 0 && j < ny) y[j] += v[k];
}

int rb_vec_scatter_add(rb_vec y, const int* idx, const double* vals, int n) {
    return guarded([&]() -> int {
        NEED(y);
        RB_REQUIRE(n >= 0, "negative count");
        RB_REQUIRE(n == 0 || (idx && vals), "null index or value pointer");
        if (n) k_vec_scatter_add<<<grid_for(n, 256), 256, 0, stream()>>>(n, y->v.get(), y->n, idx, vals);
        RB_CHECK_LAUNCH();
        return RB_OK;
    });
}

int rb_vec_scale(rb_vec y, double a) {
    return guarded([&]() -> int {
        NEED(y);
        if (y->n) k_scale<double><<<grid_for(y->n, 256), 256, 0, stream()>>>(y->n, y->v.get(), a);
        RB_CHECK_LAUNCH();
        return RB_OK;
    });
}

int rb_vec_dot(rb_vec a, rb_vec b, double* out) {
    return guarded([&]() -> int {
        NEED(a); NEED(b); NEED(out);
        RB_REQUIRE(a->n == b->n, "Cannot perform inner product: dimensions do not match");
        DevArray<double> r(1);
        dot_async(a->v.get(), b->v.get(), a->n, r.get());
        *out = read_scalar(r.get());
        return RB_OK;
    });
}

int rb_vec_norm2(rb_vec a, double* out) {
    return guarded([&]() -> int {
        NEED(a); NEED(out);
        DevArray<double> r(1);
        dot_async(a->v.get(), a->v.get(), a->n, r.get());
        *out = std::sqrt(read_scalar(r.get()));
        return RB_OK;
    });
}

// ----------------------------------------------------------- SpMV family --
int rb_spmv(rb_csr A, rb_vec x, rb_vec b) {
    return guarded([&]() -> int {
        NEED(A); NEED(x); NEED(b);
        RB_REQUIRE(x->n == A->n_cols && b->n == A->n_rows, "spmv: sizes do not match");
        spmv64(view(*A), x->v.get(), b->v.get(), handle_lanes(*A, x->v.get()));
        return RB_OK;
    });
}

int rb_residual(rb_csr A, rb_vec x, rb_vec b, rb_vec r) {
    return guarded([&]() -> int {
        NEED(A); NEED(x); NEED(b); NEED(r);
        RB_REQUIRE(x->n == A->n_cols && b->n == A->n_rows && r->n == A->n_rows,
                   "residual: sizes do not match");
        residual64(view(*A), x->v.get(), b->v.get(), r->v.get(), handle_lanes(*A, x->v.get()));
        return RB_OK;
    });
}

int rb_spmv_T(rb_csr A, rb_vec x, rb_vec b) {
    return guarded([&]() -> int {
        NEED(A); NEED(x); NEED(b);
        RB_REQUIRE(x->n == A->n_rows && b->n == A->n_cols, "spmv_T: sizes do not match");
        // a gather over A^T's pattern, cached on the handle: deterministic,
        // no atomics, no allocation after the first call
        spmv_T64(*A, x->v.get(), b->v.get());
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_spmv_append(rb_csr A, rb_vec x, rb_vec b) {
    return guarded([&]() -> int {
        NEED(A); NEED(x); NEED(b);
        RB_REQUIRE(x->n == A->n_cols && b->n == A->n_rows, "spmv_append: sizes do not match");
        spmv_append64(view(*A), x->v.get(), b->v.get(), handle_lanes(*A, x->v.get()));
        return RB_OK;
    });
}

// ---------------------------------------------------------- block CSR --
int rb_bsr_create(int n_block_rows, int n_block_cols, int b_rows, int b_cols, int64_t nnz,
                  const int* rowptr, const int* cols, const double* vals, int on_device,
                  rb_bsr* out) {
    return guarded([&]() -> int {
        ensure_device();
        NEED(out); NEED(rowptr);
        RB_REQUIRE(n_block_rows >= 0 && n_block_cols >= 0 && nnz >= 0, "negative matrix dimension");
        RB_REQUIRE(b_rows >= 1 && b_cols >= 1, "block dimensions must be at least 1");
        RB_REQUIRE((long long)n_block_rows * b_rows <= INT_MAX &&
                       (long long)n_block_cols * b_cols <= INT_MAX,
                   "scalar dimension exceeds the int32 index range");
        RB_REQUIRE(nnz <= INT_MAX, "more than 2^31-1 blocks (int32 indices)");
        RB_REQUIRE(nnz == 0 || (cols && vals), "cols/vals are NULL");
        if (!on_device) {
            RB_REQUIRE(rowptr[0] == 0 && rowptr[n_block_rows] == nnz, "rowptr does not span the blocks");
            for (int i = 0; i < n_block_rows; i++)
                RB_REQUIRE(rowptr[i] <= rowptr[i + 1], "rowptr is not monotone");
            for (int64_t j = 0; j < nnz; j++)
                RB_REQUIRE(cols[j] >= 0 && cols[j] < n_block_cols, "block column index out of range");
        }
        const size_t bs = (size_t)b_rows * b_cols;
        std::unique_ptr<rb_bsr_s> A(new rb_bsr_s());
        A->n_block_rows = n_block_rows;
        A->n_block_cols = n_block_cols;
        A->b_rows = b_rows;
        A->b_cols = b_cols;
        A->nnz = nnz;
        A->rowptr.alloc((size_t)n_block_rows + 1);
        A->cols.alloc(nnz > 0 ? (size_t)nnz : 1);
        A->vals.alloc(nnz > 0 ? (size_t)nnz * bs : 1);
        auto kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        RB_CUDA(cudaMemcpyAsync(A->rowptr.get(), rowptr, sizeof(int) * ((size_t)n_block_rows + 1),
                                kind, stream()));
        if (nnz) {
            RB_CUDA(cudaMemcpyAsync(A->cols.get(), cols, sizeof(int) * (size_t)nnz, kind, stream()));
            RB_CUDA(cudaMemcpyAsync(A->vals.get(), vals, sizeof(double) * (size_t)nnz * bs, kind,
                                    stream()));
        }
        RB_CUDA(cudaStreamSynchronize(stream()));
        *out = A.release();
        return RB_OK;
    });
}

int rb_bsr_destroy(rb_bsr A) {
    return guarded([&]() -> int {
        delete A;
        return RB_OK;
    });
}

int rb_bsr_info(rb_bsr A, int* n_block_rows, int* n_block_cols, int* b_rows, int* b_cols,
                int64_t* nnz_blocks) {
    return guarded([&]() -> int {
        NEED(A);
        if (n_block_rows) *n_block_rows = A->n_block_rows;
        if (n_block_cols) *n_block_cols = A->n_block_cols;
        if (b_rows) *b_rows = A->b_rows;
        if (b_cols) *b_cols = A->b_cols;
        if (nnz_blocks) *nnz_blocks = A->nnz;
        return RB_OK;
    });
}

int rb_bsr_download(rb_bsr A, int* rowptr, int* cols, double* vals) {
    return guarded([&]() -> int {
        NEED(A);
        if (rowptr) A->rowptr.download(rowptr, (size_t)A->n_block_rows + 1);
        if (cols) A->cols.download(cols, (size_t)A->nnz);
        if (vals) A->vals.download(vals, (size_t)A->nnz * A->b_rows * A->b_cols);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_bsr_spmv(rb_bsr A, rb_vec x, rb_vec b) {
    return guarded([&]() -> int {
        NEED(A); NEED(x); NEED(b);
        RB_REQUIRE(x->n == A->n_block_cols * A->b_cols && b->n == A->n_block_rows * A->b_rows,
                   "bsr spmv: sizes do not match");
        RB_REQUIRE(x != b, "bsr spmv: x and b must be different vectors");
        bsr_apply(*A, kBsrMult, x->v.get(), nullptr, b->v.get());
        return RB_OK;
    });
}

int rb_bsr_spmv_append(rb_bsr A, rb_vec x, rb_vec b) {
    return guarded([&]() -> int {
        NEED(A); NEED(x); NEED(b);
        RB_REQUIRE(x->n == A->n_block_cols * A->b_cols && b->n == A->n_block_rows * A->b_rows,
                   "bsr spmv_append: sizes do not match");
        RB_REQUIRE(x != b, "bsr spmv_append: x and b must be different vectors");
        bsr_apply(*A, kBsrAppend, x->v.get(), b->v.get(), b->v.get());
        return RB_OK;
    });
}

int rb_bsr_residual(rb_bsr A, rb_vec x, rb_vec b, rb_vec r) {
    return guarded([&]() -> int {
        NEED(A); NEED(x); NEED(b); NEED(r);
        RB_REQUIRE(x->n == A->n_block_cols * A->b_cols && b->n == A->n_block_rows * A->b_rows &&
                       r->n == b->n,
                   "bsr residual: sizes do not match");
        RB_REQUIRE(x != r, "bsr residual: x and r must be different vectors");
        bsr_apply(*A, kBsrResidual, x->v.get(), b->v.get(), r->v.get());
        return RB_OK;
    });
}

int rb_bsr_spmv_T(rb_bsr A, rb_vec x, rb_vec b) {
    return guarded([&]() -> int {
        NEED(A); NEED(x); NEED(b);
        RB_REQUIRE(x->n == A->n_block_rows * A->b_rows && b->n == A->n_block_cols * A->b_cols,
                   "bsr spmv_T: sizes do not match");
        RB_REQUIRE(x != b, "bsr spmv_T: x and b must be different vectors");
        bsr_spmv_T(*A, x->v.get(), b->v.get());
        return RB_OK;
    });
}

int rb_bsr_to_csr(rb_bsr A, rb_csr* out) {
    return guarded([&]() -> int {
        NEED(A); NEED(out);
        *out = bsr_to_csr(*A);
        return RB_OK;
    });
}

// --------------------------------------------------------------- gallery --
int rb_diffusion_stencil_2d(double eps, double theta, double* st) {
    return guarded([&]() -> int {
        NEED(st);
        // gallery/diffusion.hpp:58-85, same expression order
        double C = std::cos(theta), S = std::sin(theta);
        double CS = C * S, CC = C * C, SS = S * S;
        volatile double v1 = ((-1 * eps - 1) * CC + (-1 * eps - 1) * SS + (3 * eps - 3) * CS) / 6.0;
        volatile double v2 = ((2 * eps - 4) * CC + (-4 * eps + 2) * SS) / 6.0;
        volatile double v3 = ((-1 * eps - 1) * CC + (-1 * eps - 1) * SS + (-3 * eps + 3) * CS) / 6.0;
        volatile double v4 = ((-4 * eps + 2) * CC + (2 * eps - 4) * SS) / 6.0;
        volatile double v5 = ((8 * eps + 8) * CC + (8 * eps + 8) * SS) / 6.0;
        double vals[9] = {v1, v2, v3, v4, v5, v4, v3, v2, v1};
        memcpy(st, vals, sizeof(vals));
        return RB_OK;
    });
}

int rb_laplace_stencil_27pt(double* st) {
    return guarded([&]() -> int {
        NEED(st);
        for (int i = 0; i < 27; i++) st[i] = -1;
        st[13] = 26;
        return RB_OK;
    });
}

int rb_stencil_grid_impl(const double* stencil, const int* grid, int dim, rb_csr* out);

int rb_stencil_grid(const double* stencil, const int* grid, int dim, rb_csr* out) {
    return guarded([&]() -> int {
        ensure_device();
        NEED(stencil); NEED(grid); NEED(out);
        return rb_stencil_grid_impl(stencil, grid, dim, out);
    });
}

int rb_read_petsc(const char* path, rb_csr* out) {
    return guarded([&]() -> int {
        ensure_device();
        NEED(path); NEED(out);
        HostCsr H = petsc_parse(path);
        int rc = rb_csr_create(H.n_rows, H.n_cols, (int64_t)H.cols.size(), H.rowptr.data(),
                               H.cols.data(), H.vals.data(), 0, out);
        if (rc != RB_OK) return rc;
        sort_rows_diag_first(**out, false);   // finalize() sorts rows
        return RB_OK;
    });
}

int rb_petsc_read_host(const char* path, int* n_rows, int* n_cols, int64_t* nnz, int* rowptr,
                       int* cols, double* vals) {
    return guarded([&]() -> int {
        NEED(path); NEED(n_rows); NEED(n_cols); NEED(nnz);
        HostCsr H = petsc_parse(path);
        *n_rows = H.n_rows;
        *n_cols = H.n_cols;
        *nnz = (int64_t)H.cols.size();
        if (rowptr) std::copy(H.rowptr.begin(), H.rowptr.end(), rowptr);
        if (cols) std::copy(H.cols.begin(), H.cols.end(), cols);
        if (vals) std::copy(H.vals.begin(), H.vals.end(), vals);
        return RB_OK;
    });
}

int rb_petsc_write_host(const char* path, int n_rows, int n_cols, int64_t nnz, const int* rowptr,
                        const int* cols, const double* vals) {
    return guarded([&]() -> int {
        NEED(path);
        petsc_write(path, n_rows, n_cols, (long long)nnz, rowptr, cols, vals);
        return RB_OK;
    });
}

int rb_write_petsc(rb_csr A, const char* path) {
    return guarded([&]() -> int {
        NEED(A); NEED(path);
        std::vector<int> rp((size_t)A->n_rows + 1), ci((size_t)A->nnz);
        std::vector<double> cv((size_t)A->nnz);
        A->rowptr.download(rp.data(), rp.size());
        if (A->nnz) {
            A->cols.download(ci.data(), ci.size());
            A->vals.download(cv.data(), cv.size());
        }
        RB_CUDA(cudaStreamSynchronize(stream()));
        petsc_write(path, A->n_rows, A->n_cols, A->nnz, rp.data(), ci.data(), cv.data());
        return RB_OK;
    });
}

// ---------------------------------------------------------- MatrixMarket --
// read_mm / read_par_mm / write_mm (gallery/matrix_market.cpp:18-105,
// gallery/par_matrix_market.cpp:18-128); the parsing is in mmio.cu.
int rb_mm_read_host(const char* path, int mirror, int sort_rows, int* n_rows, int* n_cols,
                    int64_t* nnz, int* rowptr, int* cols, double* vals) {
    return guarded([&]() -> int {
        NEED(path); NEED(n_rows); NEED(n_cols); NEED(nnz);
        HostCsr H = mm_parse(path, mirror != 0, sort_rows != 0);
        *n_rows = H.n_rows;
        *n_cols = H.n_cols;
        *nnz = (int64_t)H.cols.size();
        if (rowptr) std::copy(H.rowptr.begin(), H.rowptr.end(), rowptr);
        if (cols) std::copy(H.cols.begin(), H.cols.end(), cols);
        if (vals) std::copy(H.vals.begin(), H.vals.end(), vals);
        return RB_OK;
    });
}

int rb_mm_write_host(const char* path, int n_rows, int n_cols, int64_t nnz, const int* rowptr,
                     const int* cols, const double* vals) {
    return guarded([&]() -> int {
        NEED(path);
        mm_write(path, n_rows, n_cols, (long long)nnz, rowptr, cols, vals);
        return RB_OK;
    });
}

static int read_mm_as(const char* path, bool par, rb_csr* out) {
    return guarded([&]() -> int {
        ensure_device();
        NEED(path); NEED(out);
        HostCsr H = mm_parse(path, par, par);
        return rb_csr_create(H.n_rows, H.n_cols, (int64_t)H.cols.size(), H.rowptr.data(),
                             H.cols.data(), H.vals.data(), 0, out);
    });
}

int rb_read_mm(const char* path, rb_csr* out) { return read_mm_as(path, false, out); }

int rb_read_par_mm(const char* path, rb_csr* out) { return read_mm_as(path, true, out); }

int rb_write_mm(rb_csr A, const char* path) {
    return guarded([&]() -> int {
        NEED(A); NEED(path);
        std::vector<int> rp((size_t)A->n_rows + 1), ci((size_t)A->nnz);
        std::vector<double> cv((size_t)A->nnz);
        A->rowptr.download(rp.data(), rp.size());
        if (A->nnz) {
            A->cols.download(ci.data(), ci.size());
            A->vals.download(cv.data(), cv.size());
        }
        RB_CUDA(cudaStreamSynchronize(stream()));
        mm_write(path, A->n_rows, A->n_cols, A->nnz, rp.data(), ci.data(), cv.data());
        return RB_OK;
    });
}

// ------------------------------------------------------ setup components --
int rb_strength(rb_csr A, int kind, double theta, rb_csr* S) {
    return guarded([&]() -> int {
        NEED(A); NEED(S);
        RB_REQUIRE(kind == RB_STRENGTH_CLASSICAL || kind == RB_STRENGTH_SYMMETRIC, "unknown strength kind");
        *S = strength(*A, kind, theta);
        return RB_OK;
    });
}

int rb_split_pmis(rb_csr S, const double* weights, int* states) {
    return guarded([&]() -> int {
        NEED(S); NEED(states);
        const int n = S->n_rows;
        std::vector<double> w = weights ? std::vector<double>(weights, weights + n) : rand_weights(n, 0);
        DevArray<double> wd((size_t)std::max(n, 1));
        wd.upload(w.data(), n);
        DevArray<int> st((size_t)std::max(n, 1));
        split_pmis(*S, wd.get(), st.get());
        st.download(states, n);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_split(rb_csr S, int kind, const double* weights, int* states) {
    return guarded([&]() -> int {
        NEED(S); NEED(states);
        RB_REQUIRE(kind >= RB_COARSEN_RS && kind <= RB_COARSEN_HMIS, "unknown coarsening kind");
        const int n = S->n_rows;
        std::vector<double> w = weights ? std::vector<double>(weights, weights + n) : rand_weights(n, 0);
        DevArray<double> wd((size_t)std::max(n, 1));
        wd.upload(w.data(), n);
        DevArray<int> st((size_t)std::max(n, 1));
        switch (kind) {
            case RB_COARSEN_RS: split_rs(*S, st.get(), true); break;
            case RB_COARSEN_CLJP: split_cljp(*S, wd.get(), st.get(), false); break;
            case RB_COARSEN_FALGOUT:
                split_rs(*S, st.get(), true);
                split_cljp(*S, wd.get(), st.get(), true);
                break;
            case RB_COARSEN_HMIS:
                split_rs(*S, st.get(), false);
                split_pmis(*S, wd.get(), st.get(), true);
                break;
            default: split_pmis(*S, wd.get(), st.get()); break;
        }
        st.download(states, n);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_interpolation(rb_csr A, rb_csr S, const int* states, int kind, double filter, rb_csr* P) {
    return guarded([&]() -> int {
        NEED(A); NEED(S); NEED(states); NEED(P);
        RB_REQUIRE(kind == RB_INTERP_DIRECT || kind == RB_INTERP_MODCLASSICAL || kind == RB_INTERP_EXTENDED,
                   "unknown interpolation kind");
        DevArray<int> st((size_t)std::max(A->n_rows, 1));
        st.upload(states, A->n_rows);
        *P = interpolation(*A, *S, st.get(), kind, filter);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_mis2(rb_csr S, const double* weights, int* states) {
    return guarded([&]() -> int {
        NEED(S); NEED(states);
        const int n = S->n_rows;
        std::vector<double> w = weights ? std::vector<double>(weights, weights + n) : rand_weights(n, 0);
        DevArray<double> wd((size_t)std::max(n, 1));
        wd.upload(w.data(), n);
        DevArray<int> st((size_t)std::max(n, 1));
        mis2(*S, wd.get(), st.get());
        st.download(states, n);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_aggregate(rb_csr A, rb_csr S, const int* states, const double* r, int* aggregates,
                 int* n_aggs) {
    return guarded([&]() -> int {
        NEED(A); NEED(S); NEED(states); NEED(aggregates); NEED(n_aggs);
        const int n = S->n_rows;
        DevArray<int> st((size_t)std::max(n, 1)), agg((size_t)std::max(n, 1));
        st.upload(states, n);
        DevArray<double> rd;
        if (r) {
            rd.alloc((size_t)std::max(n, 1));
            rd.upload(r, n);
        }
        *n_aggs = aggregate(*A, *S, st.get(), agg.get(), r ? rd.get() : nullptr);
        agg.download(aggregates, n);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_fit_candidates(int n_rows, int n_aggs, const int* aggregates, const double* B, double* R,
                      rb_csr* T) {
    return guarded([&]() -> int {
        NEED(aggregates); NEED(B); NEED(R); NEED(T);
        RB_REQUIRE(n_rows >= 0 && n_aggs >= 0, "negative size");
        ensure_device();
        DevArray<int> agg((size_t)std::max(n_rows, 1));
        agg.upload(aggregates, n_rows);
        DevArray<double> Bd((size_t)std::max(n_rows, 1)), Rd((size_t)std::max(n_aggs, 1));
        Bd.upload(B, n_rows);
        *T = fit_candidates(n_rows, n_aggs, agg.get(), Bd.get(), Rd.get());
        Rd.download(R, n_aggs);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_jacobi_prolongation(rb_csr A, rb_csr T, double omega, int steps, rb_csr* P) {
    return guarded([&]() -> int {
        NEED(A); NEED(T); NEED(P);
        RB_REQUIRE(steps >= 0, "steps < 0");
        *P = jacobi_prolongation(*A, *T, omega, steps);
        return RB_OK;
    });
}

int rb_spgemm(rb_csr A, rb_csr B, rb_csr* C) {
    return guarded([&]() -> int {
        NEED(A); NEED(B); NEED(C);
        *C = spgemm(*A, *B);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_rap(rb_csr A, rb_csr P, int diag_first, rb_csr* Ac) {
    return guarded([&]() -> int {
        NEED(A); NEED(P); NEED(Ac);
        *Ac = rap(*A, *P, nullptr, diag_first != 0);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

// ------------------------------------------------------------- hierarchy --
void rb_amg_default_opts(rb_amg_opts* o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->solver = RB_SOLVER_RS;
    o->strength_type = RB_STRENGTH_CLASSICAL;
    o->interp_type = RB_INTERP_MODCLASSICAL;
    o->relax_type = RB_RELAX_JACOBI;
    o->num_smooth_sweeps = 1;
    o->max_coarse = 50;
    o->max_levels = 25;
    o->max_iterations = 100;
    o->strong_threshold = 0.25;
    o->relax_weight = 1.0;
    o->solve_tol = 1e-7;
    o->interp_filter = 0.3;
    o->prolong_weight = 4.0 / 3.0;
    o->prolong_smooth_steps = 1;
    o->precision = RB_PREC_FP64;
    o->jacobi_compat = 0;
    o->seed_offset = 0;
    o->fuse_coarse = 1;
    o->use_graphs = 1;
    o->const_coef = 1;
    o->coarsen_type = RB_COARSEN_PMIS;
    o->num_variables = 1;
}

int rb_amg_setup(rb_csr A, const rb_amg_opts* opts, const double* weights, rb_amg* out) {
    return guarded([&]() -> int {
        rb_amg_opts o;
        if (opts) o = *opts;
        else rb_amg_default_opts(&o);
        // the options are checked before anything touches the matrix, so an
        // option this build does not have (Direct interpolation, say) is an
        // error, never a silent substitute
        RB_REQUIRE(o.solver == RB_SOLVER_RS || o.solver == RB_SOLVER_SA, "unknown solver");
        RB_REQUIRE(o.solver == RB_SOLVER_SA || o.interp_type == RB_INTERP_DIRECT ||
                       o.interp_type == RB_INTERP_MODCLASSICAL || o.interp_type == RB_INTERP_EXTENDED,
                   "interpolation must be Direct, ModClassical or Extended");
        RB_REQUIRE(o.strength_type == RB_STRENGTH_CLASSICAL || o.strength_type == RB_STRENGTH_SYMMETRIC,
                   "unknown strength type");
        RB_REQUIRE(o.relax_type == RB_RELAX_JACOBI || o.relax_type == RB_RELAX_SOR ||
                       o.relax_type == RB_RELAX_SSOR || o.relax_type == RB_RELAX_L1JACOBI,
                   "unknown relaxation type");
        RB_REQUIRE(o.precision == RB_PREC_FP64 || o.precision == RB_PREC_FP32, "unknown precision");
        RB_REQUIRE(o.coarsen_type >= RB_COARSEN_RS && o.coarsen_type <= RB_COARSEN_HMIS,
                   "unknown coarsening type");
        RB_REQUIRE(o.num_variables >= 1, "num_variables must be >= 1");
        RB_REQUIRE(o.prolong_smooth_steps >= 0, "prolong_smooth_steps < 0");
        RB_REQUIRE(o.num_smooth_sweeps >= 0, "num_smooth_sweeps < 0");
        RB_REQUIRE(o.max_levels >= 1 && o.max_coarse >= 1, "max_levels and max_coarse must be >= 1");
        NEED(A); NEED(out);
        RB_REQUIRE(A->n_rows == A->n_cols, "AMG needs a square matrix");
        std::unique_ptr<rb_amg_s> ml(new rb_amg_s());
        ml->h.setup(*A, o, weights);
        *out = ml.release();
        return RB_OK;
    });
}

int rb_amg_destroy(rb_amg ml) {
    return guarded([&]() -> int {
        delete ml;
        return RB_OK;
    });
}

int rb_amg_num_levels(rb_amg ml, int* num_levels) {
    return guarded([&]() -> int {
        NEED(ml); NEED(num_levels);
        *num_levels = ml->h.num_levels();
        return RB_OK;
    });
}

int rb_amg_level_info(rb_amg ml, int level, int* n_rows, int64_t* nnz_A, int64_t* nnz_P) {
    return guarded([&]() -> int {
        NEED(ml);
        RB_REQUIRE(level >= 0 && level < ml->h.num_levels(), "level out of range");
        const MasterLevel& M = ml->h.master[level];
        if (n_rows) *n_rows = M.A->n_rows;
        if (nnz_A) *nnz_A = M.A->nnz;
        if (nnz_P) *nnz_P = M.P ? M.P->nnz : 0;
        return RB_OK;
    });
}

int rb_amg_level_matrix(rb_amg ml, int level, int which, rb_csr* out) {
    return guarded([&]() -> int {
        NEED(ml); NEED(out);
        RB_REQUIRE(level >= 0 && level < ml->h.num_levels(), "level out of range");
        const MasterLevel& M = ml->h.master[level];
        const rb_csr_s* src = which == 0 ? M.A.get() : which == 1 ? M.P.get() : M.R.get();
        RB_REQUIRE(src != nullptr, "the coarsest level has no P/R");
        *out = clone_csr(*src);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_amg_level_states(rb_amg ml, int level, int* states) {
    return guarded([&]() -> int {
        NEED(ml); NEED(states);
        RB_REQUIRE(level >= 0 && level < ml->h.num_levels() - 1, "level has no splitting");
        const MasterLevel& M = ml->h.master[level];
        M.states.download(states, M.A->n_rows);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_amg_cycle(rb_amg ml, rb_vec x, rb_vec b) {
    return guarded([&]() -> int {
        NEED(ml); NEED(x); NEED(b);
        const int n = ml->h.master[0].A->n_rows;
        RB_REQUIRE(x->n == n && b->n == n, "cycle: vector sizes do not match");
        ml->h.cycle(x->v.get(), b->v.get(), false);
        return RB_OK;
    });
}

int rb_amg_solve(rb_amg ml, rb_vec x, rb_vec b, int* iters, double* hist, int cap) {
    return guarded([&]() -> int {
        NEED(ml); NEED(x); NEED(b);
        const int n = ml->h.master[0].A->n_rows;
        RB_REQUIRE(x->n == n && b->n == n, "solve: vector sizes do not match");
        int it = 0;
        std::vector<double> h(std::max(cap, 1));
        int rc = ml->h.solve(x->v.get(), b->v.get(), hist ? hist : h.data(), hist ? cap : 0, &it);
        if (iters) *iters = it;
        return rc;
    });
}

int rb_amg_cycle_profile(rb_amg ml, double* ms, int cap, int* n_out) {
    return guarded([&]() -> int {
        NEED(ml); NEED(ms);
        std::vector<double> v = ml->h.profile_cycle();
        const int m = std::min<int>(cap, (int)v.size());
        for (int i = 0; i < m; i++) ms[i] = v[i];
        if (n_out) *n_out = (int)v.size();
        return RB_OK;
    });
}

int rb_amg_time_operator(rb_amg ml, int level, int op, int reps, double* ms_per_launch) {
    return guarded([&]() -> int {
        NEED(ml); NEED(ms_per_launch);
        RB_REQUIRE(op >= 0 && op <= 7, "unknown operator");
        *ms_per_launch = ml->h.time_operator(level, op, reps);
        return RB_OK;
    });
}

int rb_amg_setup_seconds(rb_amg ml, double* seconds) {
    return guarded([&]() -> int {
        NEED(ml); NEED(seconds);
        *seconds = ml->h.setup_seconds;
        return RB_OK;
    });
}

int rb_amg_level_lanes(rb_amg ml, int level, int* lanes_A, int* lanes_P, int* lanes_R) {
    return guarded([&]() -> int {
        NEED(ml);
        RB_REQUIRE(level >= 0 && level < ml->h.num_levels(), "level out of range");
        int a = 0, p = 0, r = 0;
        if (ml->h.opts.precision == RB_PREC_FP32) {
            const auto& V = ml->h.lv32[level];
            a = V.dia ? 0 : V.gA; p = V.gP; r = V.gR;
        } else {
            const auto& V = ml->h.lv64[level];
            a = V.dia ? 0 : V.gA; p = V.gP; r = V.gR;
        }
        if (lanes_A) *lanes_A = a;
        if (lanes_P) *lanes_P = p;
        if (lanes_R) *lanes_R = r;
        return RB_OK;
    });
}

int rb_amg_level_storage(rb_amg ml, int level, int* ndiag) {
    return guarded([&]() -> int {
        NEED(ml); NEED(ndiag);
        RB_REQUIRE(level >= 0 && level < ml->h.num_levels(), "level out of range");
        if (ml->h.opts.precision == RB_PREC_FP32) {
            const auto& V = ml->h.lv32[level];
            *ndiag = V.dia ? V.off.nd : 0;
        } else {
            const auto& V = ml->h.lv64[level];
            *ndiag = V.dia ? V.off.nd : 0;
        }
        return RB_OK;
    });
}

int rb_amg_level_const_coef(rb_amg ml, int level, int* constant) {
    return guarded([&]() -> int {
        NEED(ml); NEED(constant);
        RB_REQUIRE(level >= 0 && level < ml->h.num_levels(), "level out of range");
        if (ml->h.opts.precision == RB_PREC_FP32) {
            const auto& V = ml->h.lv32[level];
            *constant = V.dia && V.off.mask ? (V.off.grid ? 2 : 1) : 0;
        } else {
            const auto& V = ml->h.lv64[level];
            *constant = V.dia && V.off.mask ? (V.off.grid ? 2 : 1) : 0;
        }
        return RB_OK;
    });
}

int rb_amg_level_fused_first(rb_amg ml, int level, int* fused) {
    return guarded([&]() -> int {
        NEED(ml); NEED(fused);
        RB_REQUIRE(level >= 0 && level < ml->h.num_levels(), "level out of range");
        *fused = ml->h.opts.precision == RB_PREC_FP32 ? ml->h.lv32[level].fuse_first
                                                      : ml->h.lv64[level].fuse_first;
        return RB_OK;
    });
}

int rb_amg_tail_info(rb_amg ml, int* start_level, int* ctas) {
    return guarded([&]() -> int {
        NEED(ml); NEED(start_level); NEED(ctas);
        *start_level = ml->h.tail_from;
        *ctas = ml->h.tail_from >= 0 ? ml->h.tail_ctas : 0;
        return RB_OK;
    });
}

int rb_amg_tail_timings(rb_amg ml, double* ms, int cap, int* count) {
    return guarded([&]() -> int {
        NEED(ml); NEED(count);
        const auto& t = ml->h.tail_ms;
        *count = (int)t.size();
        for (int i = 0; i < (int)t.size() && i < cap && ms; i++) ms[i] = t[i];
        return RB_OK;
    });
}

int rb_launch_count(int64_t* count) {
    return guarded([&]() -> int {
        NEED(count);
        *count = launch_counter();
        return RB_OK;
    });
}

int rb_device_alloc_count(int64_t* count) {
    return guarded([&]() -> int {
        NEED(count);
        *count = device_alloc_counter();
        return RB_OK;
    });
}

// ---------------------------------------------------------------- Krylov --
int rb_pcg(rb_csr A, rb_amg ml, rb_vec x, rb_vec b, double tol, int max_iter, int mode,
           double* hist, int cap, int* n_hist) {
    return guarded([&]() -> int {
        NEED(A); NEED(ml); NEED(x); NEED(b);
        RB_REQUIRE(x->n == A->n_cols && b->n == A->n_rows, "PCG: sizes do not match");
        RB_REQUIRE(mode == RB_PCG_REFERENCE || mode == RB_PCG_TRUE_RESIDUAL, "unknown PCG mode");
        int nh = 0;
        std::vector<double> h(1);
        int rc = ml->h.pcg(*A, x->v.get(), b->v.get(), tol, max_iter, mode, hist ? hist : h.data(),
                           hist ? cap : 0, &nh);
        if (n_hist) *n_hist = nh;
        return rc;
    });
}

int rb_fv_assemble(int nx, int ny, const double* k, rb_csr* A) {
    return guarded([&]() -> int {
        NEED(k); NEED(A);
        ensure_device();
        *A = fv_assemble(nx, ny, k);
        RB_CUDA(cudaStreamSynchronize(stream()));
        return RB_OK;
    });
}

int rb_fv_backward(int nx, int ny, const double* k, rb_csr A, const double* gA, double* gk) {
    return guarded([&]() -> int {
        NEED(k); NEED(A); NEED(gA); NEED(gk);
        fv_backward(nx, ny, k, *A, gA, gk);
        return RB_OK;
    });
}

int rb_sddmm(rb_csr A, const double* lambda, const double* x, double scale, double* out) {
    return guarded([&]() -> int {
        NEED(A); NEED(lambda); NEED(x); NEED(out);
        sddmm(*A, lambda, x, scale, out);
        return RB_OK;
    });
}

int rb_adjoint_solve(rb_csr A, rb_amg ml, rb_vec lambda, rb_vec g, double tol, int max_iter,
                     int* iters, double* relres) {
    return guarded([&]() -> int {
        NEED(A); NEED(ml); NEED(lambda); NEED(g);
        RB_REQUIRE(lambda->n == A->n_rows && g->n == A->n_rows, "adjoint: sizes do not match");
        return adjoint_solve(*A, ml->h, lambda->v.get(), g->v.get(), tol, max_iter, iters, relres);
    });
}

int rb_batch_setup(int n_sys, const rb_csr* mats, const rb_amg_opts* opts, rb_batch* out) {
    return guarded([&]() -> int {
        NEED(mats); NEED(out);
        RB_REQUIRE(n_sys >= 1, "batch: no systems");
        for (int s = 0; s < n_sys; s++) RB_REQUIRE(mats[s] != nullptr, "batch: NULL matrix");
        rb_amg_opts o;
        if (opts) o = *opts;
        else rb_amg_default_opts(&o);
        RB_REQUIRE(o.solver == RB_SOLVER_RS || o.solver == RB_SOLVER_SA, "unknown solver");
        std::vector<const rb_csr_s*> m(mats, mats + n_sys);
        *out = batch_setup(n_sys, m.data(), o);
        return RB_OK;
    });
}

int rb_batch_destroy(rb_batch B) {
    return guarded([&]() -> int {
        batch_destroy(B);
        return RB_OK;
    });
}

int rb_batch_info(rb_batch B, int* n_sys, int64_t* total_rows, int* levels) {
    return guarded([&]() -> int {
        NEED(B);
        const int n = batch_num_systems(B);
        if (n_sys) *n_sys = n;
        if (total_rows) *total_rows = batch_offset(B, n);
        if (levels) *levels = batch_packed_levels(B);
        return RB_OK;
    });
}

int rb_batch_offsets(rb_batch B, int64_t* offsets, int* levels) {
    return guarded([&]() -> int {
        NEED(B);
        const int n = batch_num_systems(B);
        for (int s = 0; s <= n; s++)
            if (offsets) offsets[s] = batch_offset(B, s);
        for (int s = 0; s < n; s++)
            if (levels) levels[s] = batch_levels(B, s);
        return RB_OK;
    });
}

int rb_batch_cycle(rb_batch B, rb_vec x, rb_vec b) {
    return guarded([&]() -> int {
        NEED(B); NEED(x); NEED(b);
        const long long N = batch_offset(B, batch_num_systems(B));
        RB_REQUIRE(x->n == N && b->n == N, "batch cycle: vector sizes do not match");
        batch_cycle(B, x->v.get(), b->v.get());
        return RB_OK;
    });
}

int rb_batch_pcg(rb_batch B, rb_vec x, rb_vec b, double tol, int max_iter, int* iters,
                 double* relres) {
    return guarded([&]() -> int {
        NEED(B); NEED(x); NEED(b); NEED(iters); NEED(relres);
        const long long N = batch_offset(B, batch_num_systems(B));
        RB_REQUIRE(x->n == N && b->n == N, "batch PCG: vector sizes do not match");
        return batch_pcg(B, x->v.get(), b->v.get(), tol, max_iter, iters, relres);
    });
}

int rb_batch_host_waits(rb_batch B, int* waits) {
    return guarded([&]() -> int {
        NEED(B); NEED(waits);
        *waits = batch_host_waits(B);
        return RB_OK;
    });
}

int rb_amg_cycle_block(rb_amg ml, rb_vec X, rb_vec B, int k) {
    return guarded([&]() -> int {
        NEED(ml); NEED(X); NEED(B);
        const long long n = ml->h.master[0].A->n_rows;
        RB_REQUIRE(k >= 2 && k <= 32, "block cycle: k must be in 2..32");
        RB_REQUIRE((long long)X->n == n * k && (long long)B->n == n * k,
                   "block cycle: X and B must hold n * k entries");
        RB_REQUIRE(ml->h.opts.relax_type == RB_RELAX_JACOBI ||
                       ml->h.opts.relax_type == RB_RELAX_L1JACOBI,
                   "block cycle: the smoother must be Jacobi or L1-Jacobi");
        ml->h.cycle_block(X->v.get(), B->v.get(), k);
        return RB_OK;
    });
}

int rb_pcg_block(rb_csr A, rb_amg ml, rb_vec X, rb_vec B, int k, double tol, int max_iter,
                 int* iters, double* relres) {
    return guarded([&]() -> int {
        NEED(A); NEED(ml); NEED(X); NEED(B); NEED(iters); NEED(relres);
        RB_REQUIRE(k >= 1 && k <= 32, "block PCG: k must be in 1..32");
        RB_REQUIRE((long long)X->n == (long long)A->n_cols * k &&
                       (long long)B->n == (long long)A->n_rows * k,
                   "block PCG: X and B must hold n * k entries");
        if (k == 1) {
            // one column: the single-vector PCG in true-residual mode
            const long mi = max_iter > 0 ? max_iter : (long)(1.3 * A->n_rows) + 2;
            std::vector<double> h((size_t)mi + 2);
            int nh = 0;
            int rc = ml->h.pcg(*A, X->v.get(), B->v.get(), tol, max_iter, RB_PCG_TRUE_RESIDUAL,
                               h.data(), (int)h.size(), &nh);
            iters[0] = std::max(nh - 1, 0);
            relres[0] = nh > 0 ? h[std::min(nh, (int)h.size()) - 1] : 0.0;
            return rc;
        }
        return ml->h.pcg_block(*A, X->v.get(), B->v.get(), k, tol, max_iter, iters, relres);
    });
}

int rb_cg(rb_csr A, rb_vec x, rb_vec b, double tol, int max_iter, double* hist, int cap,
          int* n_hist) {
    return guarded([&]() -> int {
        NEED(A); NEED(x); NEED(b);
        RB_REQUIRE(x->n == A->n_cols && b->n == A->n_rows, "CG: sizes do not match");
        int nh = 0;
        std::vector<double> h(1);
        int rc = krylov_cg(*A, x->v.get(), b->v.get(), tol, max_iter, hist ? hist : h.data(),
                           hist ? cap : 0, &nh);
        if (n_hist) *n_hist = nh;
        return rc;
    });
}

int rb_bicgstab(rb_csr A, rb_amg ml, rb_vec x, rb_vec b, double tol, int max_iter, double* hist,
                int cap, int* n_hist) {
    return guarded([&]() -> int {
        NEED(A); NEED(x); NEED(b);
        RB_REQUIRE(x->n == A->n_cols && b->n == A->n_rows, "BiCGStab: sizes do not match");
        int nh = 0;
        std::vector<double> h(1);
        int rc = krylov_bicgstab(*A, ml ? &ml->h : nullptr, x->v.get(), b->v.get(), tol, max_iter,
                                 hist ? hist : h.data(), hist ? cap : 0, &nh);
        if (n_hist) *n_hist = nh;
        return rc;
    });
}

}  // extern "C"
