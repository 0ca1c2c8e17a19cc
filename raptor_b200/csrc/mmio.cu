// mmio.cu -- MatrixMarket coordinate files <-> CSR arrays on the host.
//
// The reference reads MatrixMarket files through the NIST mmio routines
// (gallery/matrix_market.cpp:18-76 read_mm, gallery/par_matrix_market.cpp:
// 18-128 read_par_mm) and writes them with write_mm (matrix_market.cpp:
// 78-105).  Only coordinate (sparse) files are matrices there; the value
// field must be real.  Two behaviours differ between its readers and both
// are kept:
//   * read_mm builds the CSR from the entries in file order (COO_to_CSR,
//     core/matrix.cpp:285-329, a stable placement by row) and ignores the
//     symmetry field: a symmetric file yields its stored triangle only;
//   * read_par_mm also stores the mirror (j, i) of every entry of a
//     symmetric file and sorts each row by column (ParMatrix::finalize ->
//     COOMatrix::sort, core/par_matrix.cpp:111-113).
// One deliberate difference: read_par_mm adds the mirror of diagonal
// entries too, which duplicates every diagonal entry of a symmetric file;
// here a diagonal entry is stored once, so the matrix equals the full one
// (test_data/aniso.mtx then equals test_data/aniso.pm).  Beyond the
// reference, integer and pattern (value 1) fields and skew-symmetric files
// (mirror -v) are accepted; complex, hermitian and array files are refused.
// Parsing is host work (file I/O); the arrays are then uploaded once.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "rb_internal.cuh"

namespace rb {

namespace {

std::string lower(std::string s) {
    for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
    return s;
}

struct Cursor {
    const char* p;
    const char* end;
    long long line = 1;
    void skip_blank() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) p++;
    }
    // skips comment lines and empty lines, leaves p at the next data line
    void next_data_line() {
        for (;;) {
            skip_blank();
            if (p >= end) return;
            if (*p == '\n') { p++; line++; continue; }
            if (*p == '%') {
                while (p < end && *p != '\n') p++;
                continue;
            }
            return;
        }
    }
    void end_line() {
        skip_blank();
        while (p < end && *p != '\n') p++;   // tolerate trailing fields
        if (p < end) { p++; line++; }
    }
    long long integer(const char* what) {
        skip_blank();
        RB_REQUIRE(p < end && *p != '\n', std::string("MatrixMarket: missing ") + what +
                                              " on line " + std::to_string(line));
        char* q = nullptr;
        errno = 0;
        const long long v = std::strtoll(p, &q, 10);
        RB_REQUIRE(q != p && errno == 0, std::string("MatrixMarket: bad ") + what + " on line " +
                                             std::to_string(line));
        p = q;
        return v;
    }
    double real(const char* what) {
        skip_blank();
        RB_REQUIRE(p < end && *p != '\n', std::string("MatrixMarket: missing ") + what +
                                              " on line " + std::to_string(line));
        char* q = nullptr;
        const double v = std::strtod(p, &q);
        RB_REQUIRE(q != p, std::string("MatrixMarket: bad ") + what + " on line " +
                               std::to_string(line));
        p = q;
        return v;
    }
};

}  // namespace

HostCsr mm_parse(const char* path, bool mirror, bool sort_rows) {
    FILE* f = std::fopen(path, "rb");
    RB_REQUIRE(f != nullptr, std::string("cannot open ") + path);
    std::unique_ptr<FILE, int (*)(FILE*)> guard(f, std::fclose);
    std::string text;
    {
        char buf[1 << 16];
        size_t got;
        while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, got);
    }
    Cursor c{text.data(), text.data() + text.size()};

    // banner: %%MatrixMarket object format field symmetry
    const char* eol = std::find(c.p, c.end, '\n');
    const std::string banner(c.p, eol);
    RB_REQUIRE(banner.compare(0, 14, "%%MatrixMarket") == 0,
               std::string("MatrixMarket: no %%MatrixMarket banner in ") + path);
    char t[4][64] = {{0}};
    const int ntok = std::sscanf(banner.c_str() + 14, "%63s %63s %63s %63s", t[0], t[1], t[2], t[3]);
    RB_REQUIRE(ntok == 4, "MatrixMarket: banner needs object, format, field and symmetry");
    const std::string object = lower(t[0]), format = lower(t[1]), field = lower(t[2]),
                      symmetry = lower(t[3]);
    RB_REQUIRE(object == "matrix", "MatrixMarket: object '" + object + "' is not a matrix");
    RB_REQUIRE(format == "coordinate",
               "MatrixMarket: format '" + format + "' is not supported (coordinate files only)");
    RB_REQUIRE(field == "real" || field == "double" || field == "integer" || field == "pattern",
               "MatrixMarket: field '" + field + "' is not supported (real, integer, pattern)");
    RB_REQUIRE(symmetry == "general" || symmetry == "symmetric" || symmetry == "skew-symmetric",
               "MatrixMarket: symmetry '" + symmetry + "' is not supported");
    const bool pattern = field == "pattern";
    const bool sym = symmetry == "symmetric", skew = symmetry == "skew-symmetric";
    c.p = eol;

    c.next_data_line();
    const long long M = c.integer("row count"), N = c.integer("column count"),
                    nz = c.integer("entry count");
    c.end_line();
    RB_REQUIRE(M >= 0 && N >= 0 && M <= INT_MAX && N <= INT_MAX && nz >= 0,
               "MatrixMarket: bad size line");

    std::vector<int> ri, ci;
    std::vector<double> v;
    const bool mirrored = mirror && (sym || skew);
    const size_t cap = (size_t)nz * (mirrored ? 2 : 1);
    ri.reserve(cap);
    ci.reserve(cap);
    v.reserve(cap);
    for (long long k = 0; k < nz; k++) {
        c.next_data_line();
        RB_REQUIRE(c.p < c.end, "MatrixMarket: file ends after " + std::to_string(k) + " of " +
                                    std::to_string(nz) + " entries");
        const long long i = c.integer("row index"), j = c.integer("column index");
        const double val = pattern ? 1.0 : c.real("value");
        c.end_line();
        RB_REQUIRE(i >= 1 && i <= M && j >= 1 && j <= N,
                   "MatrixMarket: entry " + std::to_string(k + 1) + " (" + std::to_string(i) +
                       ", " + std::to_string(j) + ") outside the " + std::to_string(M) + " x " +
                       std::to_string(N) + " matrix");
        ri.push_back((int)(i - 1));
        ci.push_back((int)(j - 1));
        v.push_back(val);
        if (mirrored && i != j) {
            RB_REQUIRE(j <= M && i <= N, "MatrixMarket: symmetric file that is not square");
            ri.push_back((int)(j - 1));
            ci.push_back((int)(i - 1));
            v.push_back(skew ? -val : val);
        }
    }
    RB_REQUIRE(ri.size() <= (size_t)INT_MAX, "MatrixMarket: more than 2^31-1 nonzeros");

    // stable placement by row (file order within a row)
    HostCsr A;
    A.n_rows = (int)M;
    A.n_cols = (int)N;
    const size_t nnz = ri.size();
    A.rowptr.assign((size_t)M + 1, 0);
    for (size_t e = 0; e < nnz; e++) A.rowptr[(size_t)ri[e] + 1]++;
    for (long long r = 0; r < M; r++) A.rowptr[(size_t)r + 1] += A.rowptr[(size_t)r];
    A.cols.resize(nnz);
    A.vals.resize(nnz);
    std::vector<int> at(A.rowptr.begin(), A.rowptr.end() - 1);
    for (size_t e = 0; e < nnz; e++) {
        const int d = at[(size_t)ri[e]]++;
        A.cols[(size_t)d] = ci[e];
        A.vals[(size_t)d] = v[e];
    }
    if (sort_rows) {
        std::vector<std::pair<int, double>> row;
        for (long long r = 0; r < M; r++) {
            const int s = A.rowptr[(size_t)r], e = A.rowptr[(size_t)r + 1];
            row.clear();
            for (int q = s; q < e; q++) row.emplace_back(A.cols[(size_t)q], A.vals[(size_t)q]);
            std::stable_sort(row.begin(), row.end(),
                             [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
                                 return a.first < b.first;
                             });
            for (int q = s; q < e; q++) {
                A.cols[(size_t)q] = row[(size_t)(q - s)].first;
                A.vals[(size_t)q] = row[(size_t)(q - s)].second;
            }
        }
    }
    return A;
}

// write_mm (gallery/matrix_market.cpp:78-105): a coordinate real general
// file, one "%" comment line, "M N nnz", then "i j value" per entry in row
// order, 1-based, values as %2.15e.
void mm_write(const char* path, int n_rows, int n_cols, long long nnz, const int* rowptr,
              const int* cols, const double* vals) {
    RB_REQUIRE(n_rows >= 0 && n_cols >= 0 && nnz >= 0, "negative matrix dimension");
    RB_REQUIRE(n_rows == 0 || (rowptr && (nnz == 0 || (cols && vals))), "missing CSR arrays");
    RB_REQUIRE(n_rows == 0 || (rowptr[0] == 0 && rowptr[n_rows] == nnz),
               "row pointers do not span the nonzeros");
    FILE* f = std::fopen(path, "w");
    RB_REQUIRE(f != nullptr, std::string("cannot write ") + path);
    std::unique_ptr<FILE, int (*)(FILE*)> guard(f, std::fclose);
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%%\n");
    std::fprintf(f, "%d %d %lld\n", n_rows, n_cols, nnz);
    for (int i = 0; i < n_rows; i++)
        for (int q = rowptr[i]; q < rowptr[i + 1]; q++)
            std::fprintf(f, "%d %d %2.15e\n", i + 1, cols[q] + 1, vals[q]);
    RB_REQUIRE(std::ferror(f) == 0, std::string("write failed: ") + path);
}

}  // namespace rb
