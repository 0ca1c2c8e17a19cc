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
#include <cstdint>
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

// ---------------------------------------------------------------- PETSc --
// PETSc's binary AIJ matrix format (what MatView writes to a binary viewer
// and MatLoad reads; the reference's readMatrix / readParMatrix input,
// gallery/matrix_IO.cpp:24-110, gallery/par_matrix_IO.cpp:22+): big-endian
// int32 header (1211216, rows, columns, nonzeros), int32 row lengths, int32
// column indices, float64 values, rows in order and each row's entries as
// stored.
namespace {
constexpr int kPetscMatCode = 1211216;

void put_be32(unsigned char* p, unsigned v) {
    p[0] = (unsigned char)(v >> 24);
    p[1] = (unsigned char)(v >> 16);
    p[2] = (unsigned char)(v >> 8);
    p[3] = (unsigned char)v;
}
}  // namespace

HostCsr petsc_parse(const char* path) {
    FILE* f = std::fopen(path, "rb");
    RB_REQUIRE(f != nullptr, std::string("cannot open ") + path);
    std::unique_ptr<FILE, int (*)(FILE*)> guard(f, std::fclose);
    auto be32 = [&](int* dst, size_t n) {
        std::vector<unsigned char> buf(4 * n);
        RB_REQUIRE(std::fread(buf.data(), 1, buf.size(), f) == buf.size(), "truncated PETSc file");
        for (size_t i = 0; i < n; i++)
            dst[i] = (int)((unsigned)buf[4 * i] << 24 | (unsigned)buf[4 * i + 1] << 16 |
                           (unsigned)buf[4 * i + 2] << 8 | (unsigned)buf[4 * i + 3]);
    };
    int hdr[4];
    be32(hdr, 4);
    RB_REQUIRE(hdr[0] == kPetscMatCode, "not a PETSc binary AIJ matrix");
    HostCsr A;
    A.n_rows = hdr[1];
    A.n_cols = hdr[2];
    const int nnz = hdr[3];
    RB_REQUIRE(A.n_rows >= 0 && A.n_cols >= 0 && nnz >= 0, "negative size in a PETSc header");
    std::vector<int> lens((size_t)A.n_rows);
    be32(lens.data(), lens.size());
    A.rowptr.assign((size_t)A.n_rows + 1, 0);
    for (int i = 0; i < A.n_rows; i++) {
        RB_REQUIRE(lens[i] >= 0, "negative row length in a PETSc file");
        A.rowptr[i + 1] = A.rowptr[i] + lens[i];
        RB_REQUIRE(A.rowptr[i + 1] <= nnz, "PETSc row lengths exceed the nonzero count");
    }
    RB_REQUIRE(A.rowptr[A.n_rows] == nnz, "PETSc row lengths do not add up to the nonzero count");
    A.cols.resize((size_t)nnz);
    be32(A.cols.data(), A.cols.size());
    for (int c : A.cols) RB_REQUIRE(c >= 0 && c < A.n_cols, "PETSc column index out of range");
    A.vals.resize((size_t)nnz);
    std::vector<unsigned char> buf(8 * (size_t)nnz);
    RB_REQUIRE(std::fread(buf.data(), 1, buf.size(), f) == buf.size(), "truncated PETSc file");
    for (int j = 0; j < nnz; j++) {
        uint64_t u = 0;
        for (int k = 0; k < 8; k++) u = (u << 8) | buf[8 * (size_t)j + k];
        std::memcpy(&A.vals[j], &u, 8);
    }
    return A;
}

void petsc_write(const char* path, int n_rows, int n_cols, long long nnz, const int* rowptr,
                 const int* cols, const double* vals) {
    RB_REQUIRE(n_rows >= 0 && n_cols >= 0 && nnz >= 0, "negative matrix dimension");
    RB_REQUIRE(nnz <= INT_MAX, "more nonzeros than a PETSc binary AIJ file holds");
    RB_REQUIRE(n_rows == 0 || (rowptr && (nnz == 0 || (cols && vals))), "missing CSR arrays");
    RB_REQUIRE(n_rows == 0 || (rowptr[0] == 0 && rowptr[n_rows] == nnz),
               "row pointers do not span the nonzeros");
    std::vector<unsigned char> out(16 + 4 * (size_t)n_rows + 12 * (size_t)nnz);
    unsigned char* p = out.data();
    put_be32(p, (unsigned)kPetscMatCode);
    put_be32(p + 4, (unsigned)n_rows);
    put_be32(p + 8, (unsigned)n_cols);
    put_be32(p + 12, (unsigned)nnz);
    p += 16;
    for (int i = 0; i < n_rows; i++, p += 4) {
        RB_REQUIRE(rowptr[i + 1] >= rowptr[i], "row pointers decrease");
        put_be32(p, (unsigned)(rowptr[i + 1] - rowptr[i]));
    }
    for (long long j = 0; j < nnz; j++, p += 4) {
        RB_REQUIRE(cols[j] >= 0 && cols[j] < n_cols, "column index out of range");
        put_be32(p, (unsigned)cols[j]);
    }
    for (long long j = 0; j < nnz; j++, p += 8) {
        uint64_t u;
        std::memcpy(&u, &vals[j], 8);
        for (int k = 0; k < 8; k++) p[k] = (unsigned char)(u >> (56 - 8 * k));
    }
    FILE* f = std::fopen(path, "wb");
    RB_REQUIRE(f != nullptr, std::string("cannot write ") + path);
    std::unique_ptr<FILE, int (*)(FILE*)> guard(f, std::fclose);
    RB_REQUIRE(std::fwrite(out.data(), 1, out.size(), f) == out.size(),
               std::string("write failed: ") + path);
}

}  // namespace rb
