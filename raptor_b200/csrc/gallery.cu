// gallery.cu -- par_stencil_grid on the device (gallery/par_stencil.hpp:16-236).
//
// The reference builds one data array per nonzero stencil entry, zeroes
// boundary runs of it (:137-209), and gives row i's entry d the value of the
// mirrored entry Ns-1-d at position i (:220).  The zeroing loops reduce to a
// closed form: for entry s and each dimension j where its offset o is
// nonzero, with len_j = prod_{k < dim-j-1} grid[k] and step_j = len_j*grid[0],
// position p is zeroed when o > 0 and p mod step_j < len_j, or when o < 0 and
// p mod step_j >= step_j - len_j.  Each row is then generated independently.
#include <cmath>
#include <memory>
#include <vector>

#include "rb_internal.cuh"

namespace rb {

struct StencilDesc {
    int dim, ns;
    long long n;
    long long diag[27];
    double val[27];
    int off[27][3];
    long long len[3], step[3];
};

__device__ __forceinline__ bool stencil_kept(const StencilDesc& d, int s, long long p) {
    for (int j = 0; j < d.dim; j++) {
        const int o = d.off[s][j];
        if (o == 0) continue;
        const long long m = p % d.step[j];
        if (o > 0 && m < d.len[j]) return false;
        if (o < 0 && m >= d.step[j] - d.len[j]) return false;
    }
    return true;
}

template <bool FILL>
__global__ void k_stencil_rows(StencilDesc d, int* cnt, const int* rp, int* ci, double* cv) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    int k = 0, out = FILL ? rp[i] : 0;
    for (int e = 0; e < d.ns; e++) {
        const long long col = d.diag[e] + i;
        if (col < 0 || col >= d.n) continue;
        const int s = d.ns - e - 1;
        const double v = stencil_kept(d, s, i) ? d.val[s] : 0.0;
        if (fabs(v) > 1e-16) {
            if (FILL) { ci[out + k] = (int)col; cv[out + k] = v; }
            k++;
        }
    }
    if (!FILL) cnt[i] = k;
}

}  // namespace rb

using namespace rb;

extern "C" int rb_stencil_grid_impl(const double* stencil, const int* grid, int dim, rb_csr* out) {
    RB_REQUIRE(dim >= 1 && dim <= 3, "stencil dimension must be 1, 2 or 3");
    StencilDesc d{};
    d.dim = dim;
    int slen = 1;
    d.n = 1;
    for (int j = 0; j < dim; j++) {
        RB_REQUIRE(grid[j] > 0, "grid sizes must be positive");
        slen *= 3;
        d.n *= grid[j];
    }
    RB_REQUIRE(d.n <= INT_MAX, "grid has more than 2^31-1 points");
    long long strides[3];
    strides[0] = 1;
    for (int i = 0; i < dim - 1; i++) strides[i + 1] = grid[dim - i - 1] * strides[i];
    int ns = 0;
    for (int s = 0; s < slen; s++) {
        if (std::fabs(stencil[s]) > 1e-16) {
            int p = 1;
            for (int j = 0; j < dim; j++) {
                d.off[ns][dim - j - 1] = ((s / p) % 3) - 1;
                p *= 3;
            }
            d.val[ns] = stencil[s];
            ns++;
        }
    }
    d.ns = ns;
    for (int e = 0; e < ns; e++) {
        d.diag[e] = 0;
        for (int i = 0; i < dim; i++) d.diag[e] += strides[i] * d.off[e][dim - i - 1];
    }
    for (int j = 0; j < dim; j++) {
        long long len = 1;
        for (int k = 0; k < dim - j - 1; k++) len *= grid[k];
        d.len[j] = len;
        d.step[j] = len * grid[0];
    }
    const int n = (int)d.n;
    DevArray<int> cnt((size_t)n + 1);
    k_stencil_rows<false><<<grid_for(n, 256), 256, 0, stream()>>>(d, cnt.get(), nullptr, nullptr, nullptr);
    RB_CHECK_LAUNCH();
    DevArray<int> rp((size_t)n + 1);
    long long nnz = exclusive_scan(cnt.get(), rp.get(), n);
    std::unique_ptr<rb_csr_s> A(new_csr(n, n, nnz));
    A->rowptr = std::move(rp);
    k_stencil_rows<true><<<grid_for(n, 256), 256, 0, stream()>>>(d, nullptr, A->rowptr.get(),
                                                                A->cols.get(), A->vals.get());
    RB_CHECK_LAUNCH();
    RB_CUDA(cudaStreamSynchronize(stream()));
    *out = A.release();
    return RB_OK;
}
