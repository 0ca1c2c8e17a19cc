// Host build of the per-row direct interpolation that the CUDA kernels run
// (raptor_b200/csrc/direct_interp.cuh), for a CPU test against the
// restatement: count pass, prefix sum, fill pass, as the kernels do.
#include "direct_interp.cuh"

extern "C" int direct_rows_count(int n, const int* srp, const int* sci, const int* st, int* rp) {
    rp[0] = 0;
    for (int i = 0; i < n; i++) rp[i + 1] = rp[i] + rb::direct_row_count(i, srp, sci, st);
    return rp[n];
}

extern "C" void direct_rows_fill(int n, const int* arp, const int* aci, const double* acv,
                                 const int* srp, const int* sci, const int* st, const int* rp,
                                 int* pcols, double* pvals) {
    for (int i = 0; i < n; i++) rb::direct_row_fill(i, arp, aci, acv, srp, sci, st, rp[i], pcols, pvals);
}
