// direct_interp.cuh -- direct interpolation, one fine row at a time.
//
// direct_interpolation (ruge_stuben/par_interpolation.cpp:1453-1715, world
// size 1).  A and S are sorted with the diagonal first, then by column (the
// reference sorts and moves the diagonal, :1466-1469; every level of the
// hierarchy is stored that way).  Row i of P:
//   * C point: the identity entry;
//   * otherwise, over the strong C neighbours c of i (S's row in order,
//     skipping its diagonal entry) with a_ic their A values: sum them by sign
//     (sum_strong_neg, sum_strong_pos); sum every off-diagonal a_ij by sign
//     (sum_all_neg, sum_all_pos); alpha = sum_all_neg / sum_strong_neg and,
//     when no strong C neighbour is positive, a_ii += sum_all_pos and
//     beta = 0, else beta = sum_all_pos / sum_strong_pos; then
//     w_ic = -alpha / a_ii * a_ic for a_ic < 0, -beta / a_ii * a_ic else.
// A row without a negative strong C neighbour divides by zero in alpha, as
// the reference does (:1645), and no entry of the row uses the quotient.
// The A value at a strong position is found by walking A's row forward in
// step with S's (:1476-1490); the walk stops at the row's end, so an S entry
// without an A entry reads 0 instead of running past the row.
//
// The same functions run in the CUDA kernels (one thread per row) and in a
// host build that tests them against the CPU restatement.
#pragma once

#if defined(__CUDACC__)
#define RB_HD __host__ __device__
#else
#define RB_HD
#endif

namespace rb {

constexpr int kDirectSelected = 1;   // C point (the C/F state of PMIS)

// Entries of row i of P: 1 for a C point, else its strong C neighbours.
RB_HD inline int direct_row_count(int i, const int* srp, const int* sci, const int* st) {
    if (st[i] == kDirectSelected) return 1;
    int s = srp[i];
    const int e = srp[i + 1];
    if (s < e && sci[s] == i) s++;
    int k = 0;
    for (int j = s; j < e; j++) k += st[sci[j]] == kDirectSelected;
    return k;
}

// Writes row i of P from position p0: fine column indices (mapped to coarse
// indices afterwards) and weights.
RB_HD inline void direct_row_fill(int i, const int* arp, const int* aci, const double* acv,
                                  const int* srp, const int* sci, const int* st, int p0,
                                  int* pcols, double* pvals) {
    if (st[i] == kDirectSelected) {
        pcols[p0] = i;
        pvals[p0] = 1.0;
        return;
    }
    int s = srp[i];
    const int e = srp[i + 1];
    if (s < e && sci[s] == i) s++;
    const int a0 = arp[i], a1 = arp[i + 1];
    double sum_strong_pos = 0, sum_strong_neg = 0;
    int nstrong = 0;
    int ctr = a0;
    for (int j = s; j < e; j++) {
        const int col = sci[j];
        while (ctr < a1 && aci[ctr] != col) ctr++;
        if (st[col] == kDirectSelected) {
            const double val = ctr < a1 ? acv[ctr] : 0.0;
            if (val < 0) sum_strong_neg += val;
            else sum_strong_pos += val;
            nstrong++;
        }
    }
    if (nstrong == 0) return;   // nothing to write (and A's row may be empty)
    double diag = a0 < a1 ? acv[a0] : 0.0;
    double sum_all_pos = 0, sum_all_neg = 0;
    for (int j = a0 + 1; j < a1; j++) {
        const double val = acv[j];
        if (val < 0) sum_all_neg += val;
        else sum_all_pos += val;
    }
    const double alpha = sum_all_neg / sum_strong_neg;
    double beta;
    if (sum_strong_pos == 0) {
        diag += sum_all_pos;
        beta = 0;
    } else {
        beta = sum_all_pos / sum_strong_pos;
    }
    const double neg_coeff = -alpha / diag;
    const double pos_coeff = -beta / diag;
    int m = p0;
    ctr = a0;
    for (int j = s; j < e; j++) {
        const int col = sci[j];
        while (ctr < a1 && aci[ctr] != col) ctr++;
        if (st[col] == kDirectSelected) {
            const double val = ctr < a1 ? acv[ctr] : 0.0;
            pcols[m] = col;
            pvals[m] = val < 0 ? neg_coeff * val : pos_coeff * val;
            m++;
        }
    }
}

}  // namespace rb
