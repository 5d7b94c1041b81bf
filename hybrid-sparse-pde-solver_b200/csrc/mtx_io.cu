// mtx_io.cu -- MatrixMarket (.mtx) files: the on-disk format that feeds the engine.
//
// Host code.  Same accepted formats and the same conversions as the reference's
// MatrixMarketIO (include/utils/matrix_market_io.hpp:80-130, src/utils/matrix_market_io.cpp):
//   matrices  "%%MatrixMarket matrix coordinate real|integer|pattern general|symmetric|
//             skew-symmetric|hermitian"; 1-based indices; pattern entries are 1.0;
//             symmetric storage mirrors every off-diagonal entry, skew-symmetric mirrors it
//             negated (hermitian is read as stored); complex fields and the array format are
//             refused; reading stops after the header's entry count.  The CSR is built like
//             SparseMatrix::from_coo (sparse_matrix.cpp:242-282): entries sorted by (row,
//             column), duplicates summed (here in file order: the reference's unstable sort
//             leaves their order unspecified).
//   vectors   array format ("rows cols" size line, values in order) or coordinate ("N",
//             "N 1" or "N 1 nnz" size line, "index value" lines); without a banner the first
//             line is skipped, as the reference's reader does; when expected_n is given and
//             the count differs, the result is expected_n ones (the reference resizes with
//             Vector::resize, which assigns).
//   writing   "%.15e" values, a "% comment" line when a comment is given.
// The parser reads the whole file at once and converts numbers with strtol / strtod.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"

namespace {

int fail(int code, const std::string& m) { return hamlss::set_last_error(code, m); }

enum Fmt { COORD = 0, ARRAY = 1 };
enum Field { REAL = 0, INTEGER = 1, COMPLEX = 2, PATTERN = 3 };
enum Sym { GENERAL = 0, SYMMETRIC = 1, SKEW = 2, HERMITIAN = 3 };

struct Header {
    int fmt = COORD, field = REAL, sym = GENERAL;
    long long rows = 0, cols = 0, nnz = 0;
};

bool read_file(const char* path, std::string& out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(sz > 0 ? (size_t)sz : 0);
    const size_t got = sz > 0 ? std::fread(&out[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    out.resize(got);
    return true;
}

// Line cursor over the file contents.
struct Lines {
    const std::string& s;
    size_t p = 0;
    explicit Lines(const std::string& str) : s(str) {}
    bool next(const char** b, const char** e) {
        if (p >= s.size()) return false;
        size_t q = s.find('\n', p);
        if (q == std::string::npos) q = s.size();
        *b = s.data() + p;
        *e = s.data() + q;
        if (*e > *b && (*e)[-1] == '\r') --*e;
        p = q + 1;
        return true;
    }
    // next line that is neither empty nor a comment
    bool data(const char** b, const char** e) {
        while (next(b, e))
            if (*e > *b && **b != '%') return true;
        return false;
    }
};

std::string lower(std::string t) {
    for (auto& c : t) c = (char)std::tolower((unsigned char)c);
    return t;
}

int parse_banner(const char* b, const char* e, Header* h) {
    std::vector<std::string> tok;
    std::string cur;
    for (const char* q = b; q <= e; ++q) {
        if (q == e || std::isspace((unsigned char)*q)) {
            if (!cur.empty()) tok.push_back(lower(cur));
            cur.clear();
        } else {
            cur += *q;
        }
    }
    if (tok.size() < 5) return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: invalid header");
    if (tok[2] == "coordinate") h->fmt = COORD;
    else if (tok[2] == "array") h->fmt = ARRAY;
    else return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: unknown format " + tok[2]);
    if (tok[3] == "real") h->field = REAL;
    else if (tok[3] == "integer") h->field = INTEGER;
    else if (tok[3] == "complex") h->field = COMPLEX;
    else if (tok[3] == "pattern") h->field = PATTERN;
    else return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: unknown field " + tok[3]);
    if (tok[4] == "general") h->sym = GENERAL;
    else if (tok[4] == "symmetric") h->sym = SYMMETRIC;
    else if (tok[4] == "skew-symmetric") h->sym = SKEW;
    else if (tok[4] == "hermitian") h->sym = HERMITIAN;
    else return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: unknown symmetry " + tok[4]);
    return HAMLSS_OK;
}

// Up to `max` integers from [b, e); returns how many were read.
int ints(const char* b, const char* e, long long* out, int max) {
    std::string line(b, e);
    const char* q = line.c_str();
    int k = 0;
    while (k < max) {
        char* end = nullptr;
        errno = 0;
        const long long v = std::strtoll(q, &end, 10);
        if (end == q || errno) break;
        out[k++] = v;
        q = end;
    }
    return k;
}

struct Coo {
    long long rows = 0, cols = 0;
    std::vector<int> r, c;
    std::vector<double> v;
};

int load_coo(const char* path, Coo* coo) {
    std::string text;
    if (!read_file(path, text))
        return fail(HAMLSS_ERR_INVALID, std::string("MatrixMarket: cannot open '") + path + "'");
    Lines L(text);
    const char *b, *e;
    if (!L.next(&b, &e) || e - b < 2 || b[0] != '%' || b[1] != '%')
        return fail(HAMLSS_ERR_MALFORMED, std::string("MatrixMarket: missing %% banner in ") + path);
    Header h;
    int rc = parse_banner(b, e, &h);
    if (rc) return rc;
    if (h.fmt != COORD)
        return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: a matrix must be in coordinate format");
    if (h.field == COMPLEX) return fail(HAMLSS_ERR_INVALID, "MatrixMarket: complex matrices are not supported");
    long long sz[3] = {0, 0, 0};
    if (!L.data(&b, &e) || ints(b, e, sz, 3) < 3)
        return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: missing size line");
    if (sz[0] < 0 || sz[1] < 0 || sz[2] < 0 || sz[0] > 0x7fffffff || sz[1] > 0x7fffffff)
        return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: bad size line");
    coo->rows = sz[0];
    coo->cols = sz[1];
    const long long nnz = sz[2];
    const size_t reserve = (size_t)(h.sym == GENERAL ? nnz : 2 * nnz);
    coo->r.reserve(reserve);
    coo->c.reserve(reserve);
    coo->v.reserve(reserve);
    long long got = 0;
    std::string line;
    while (got < nnz && L.data(&b, &e)) {
        line.assign(b, e);
        const char* q = line.c_str();
        char* end = nullptr;
        long long r = std::strtoll(q, &end, 10);
        if (end == q) return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: bad entry line");
        q = end;
        long long c = std::strtoll(q, &end, 10);
        if (end == q) return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: bad entry line");
        q = end;
        double v = 1.0;
        if (h.field != PATTERN) {
            v = std::strtod(q, &end);
            if (end == q) return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: bad entry value");
        }
        --r;
        --c;
        if (r < 0 || r >= coo->rows || c < 0 || c >= coo->cols)
            return fail(HAMLSS_ERR_MALFORMED, "MatrixMarket: entry index out of range");
        coo->r.push_back((int)r);
        coo->c.push_back((int)c);
        coo->v.push_back(v);
        if ((h.sym == SYMMETRIC || h.sym == SKEW) && r != c) {
            coo->r.push_back((int)c);
            coo->c.push_back((int)r);
            coo->v.push_back(h.sym == SYMMETRIC ? v : -v);
        }
        ++got;
    }
    return HAMLSS_OK;
}

struct CsrHost {
    int rows = 0, cols = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
};

// SparseMatrix::from_coo: sort by (row, column), sum duplicates.
void coo_to_csr(const Coo& coo, CsrHost* out) {
    const size_t nz = coo.r.size();
    std::vector<size_t> order(nz);
    std::iota(order.begin(), order.end(), (size_t)0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        if (coo.r[a] != coo.r[b]) return coo.r[a] < coo.r[b];
        return coo.c[a] < coo.c[b];
    });
    out->rows = (int)coo.rows;
    out->cols = (int)coo.cols;
    out->rp.assign((size_t)coo.rows + 1, 0);
    out->ci.clear();
    out->v.clear();
    out->ci.reserve(nz);
    out->v.reserve(nz);
    int last_r = -1, last_c = -1;
    for (size_t p = 0; p < nz; ++p) {
        const size_t o = order[p];
        const int r = coo.r[o], c = coo.c[o];
        if (r == last_r && c == last_c) {
            out->v.back() += coo.v[o];
        } else {
            out->ci.push_back(c);
            out->v.push_back(coo.v[o]);
            out->rp[(size_t)r + 1]++;
            last_r = r;
            last_c = c;
        }
    }
    for (size_t i = 0; i < (size_t)coo.rows; ++i) out->rp[i + 1] += out->rp[i];
}

int load_csr(const char* path, CsrHost* out) {
    Coo coo;
    int rc = load_coo(path, &coo);
    if (rc) return rc;
    if (coo.r.size() > 0x7fffffffu) return fail(HAMLSS_ERR_NOMEM, "MatrixMarket: too many entries");
    coo_to_csr(coo, out);
    return HAMLSS_OK;
}

}  // namespace

extern "C" {

int hamlss_mtx_read_header(const char* path, int32_t* format, int32_t* field, int32_t* symmetry,
                           int64_t* rows, int64_t* cols, int64_t* entries) {
    if (!path) return fail(HAMLSS_ERR_INVALID, "null path");
    std::string text;
    if (!read_file(path, text))
        return fail(HAMLSS_ERR_INVALID, std::string("MatrixMarket: cannot open '") + path + "'");
    Lines L(text);
    const char *b, *e;
    if (!L.next(&b, &e) || e - b < 2 || b[0] != '%' || b[1] != '%')
        return fail(HAMLSS_ERR_MALFORMED, std::string("MatrixMarket: missing %% banner in ") + path);
    Header h;
    int rc = parse_banner(b, e, &h);
    if (rc) return rc;
    long long sz[3] = {0, 0, 0};
    if (L.data(&b, &e)) ints(b, e, sz, 3);
    if (h.fmt == ARRAY) sz[2] = sz[0] * sz[1];
    if (format) *format = h.fmt;
    if (field) *field = h.field;
    if (symmetry) *symmetry = h.sym;
    if (rows) *rows = sz[0];
    if (cols) *cols = sz[1];
    if (entries) *entries = sz[2];
    return HAMLSS_OK;
}

int hamlss_mtx_read_matrix(const char* path, int32_t* rows, int32_t* cols, int32_t* nnz, int32_t* row_ptr,
                           int32_t* col_idx, double* values) {
    if (!path || !rows || !cols || !nnz) return fail(HAMLSS_ERR_INVALID, "null argument");
    CsrHost A;
    int rc = load_csr(path, &A);
    if (rc) return rc;
    *rows = A.rows;
    *cols = A.cols;
    *nnz = (int32_t)A.ci.size();
    if (row_ptr) std::memcpy(row_ptr, A.rp.data(), sizeof(int32_t) * A.rp.size());
    if (col_idx && !A.ci.empty()) std::memcpy(col_idx, A.ci.data(), sizeof(int32_t) * A.ci.size());
    if (values && !A.v.empty()) std::memcpy(values, A.v.data(), sizeof(double) * A.v.size());
    return HAMLSS_OK;
}

int hamlss_mtx_read_vector(const char* path, int32_t expected_n, double* values, int32_t* n) {
    if (!path || !n) return fail(HAMLSS_ERR_INVALID, "null argument");
    std::string text;
    if (!read_file(path, text))
        return fail(HAMLSS_ERR_INVALID, std::string("MatrixMarket: cannot open '") + path + "'");
    Lines L(text);
    const char *b, *e;
    Header h;   // coordinate unless a banner says otherwise
    if (L.next(&b, &e) && e - b >= 2 && b[0] == '%' && b[1] == '%') {
        int rc = parse_banner(b, e, &h);
        if (rc) return rc;
    }
    long long entries = 0;
    bool found = false;
    if (L.data(&b, &e)) {
        long long sz[3] = {0, 0, 0};
        const int k = ints(b, e, sz, 3);
        if (h.fmt == ARRAY) entries = sz[0] * sz[1];
        else entries = (k >= 3) ? sz[2] : sz[0];
        found = k > 0;
    }
    if (expected_n > 0 && !found) entries = expected_n;
    std::vector<double> out((size_t)std::max<long long>(entries > 0 ? entries : expected_n, 0), 0.0);
    size_t idx = 0;
    std::string line;
    while (L.data(&b, &e)) {
        line.assign(b, e);
        const char* q = line.c_str();
        char* end = nullptr;
        if (h.fmt == COORD) {
            const long long r = std::strtoll(q, &end, 10);
            if (end == q) continue;
            q = end;
            const double v = std::strtod(q, &end);
            if (end == q) continue;
            if (r - 1 >= 0 && (size_t)(r - 1) < out.size()) out[(size_t)(r - 1)] = v;
        } else {
            const double v = std::strtod(q, &end);
            if (end != q && idx < out.size()) out[idx++] = v;
        }
    }
    // a size other than expected_n gives expected_n ones: the reference's Vector::resize
    // (vector.cpp:26-28) assigns rather than pads
    if (expected_n > 0 && out.size() != (size_t)expected_n) out.assign((size_t)expected_n, 1.0);
    *n = (int32_t)out.size();
    if (values && !out.empty()) std::memcpy(values, out.data(), sizeof(double) * out.size());
    return HAMLSS_OK;
}

int hamlss_mtx_write_vector(const char* path, int32_t n, const double* values, const char* comment) {
    if (!path || n < 0 || (n && !values)) return fail(HAMLSS_ERR_INVALID, "bad arguments");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(HAMLSS_ERR_INVALID, std::string("MatrixMarket: cannot write to '") + path + "'");
    std::fprintf(f, "%%%%MatrixMarket matrix array real general\n");
    if (comment && *comment) std::fprintf(f, "%% %s\n", comment);
    std::fprintf(f, "%d 1\n", n);
    for (int32_t i = 0; i < n; ++i) std::fprintf(f, "%.15e\n", values[i]);
    std::fclose(f);
    return HAMLSS_OK;
}

int hamlss_mtx_write_matrix(const char* path, int32_t rows, int32_t cols, int32_t nnz, const int32_t* row_ptr,
                            const int32_t* col_idx, const double* values, const char* comment) {
    if (!path || rows < 0 || cols < 0 || nnz < 0 || !row_ptr || (nnz && (!col_idx || !values)))
        return fail(HAMLSS_ERR_INVALID, "bad arguments");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(HAMLSS_ERR_INVALID, std::string("MatrixMarket: cannot write to '") + path + "'");
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n");
    if (comment && *comment) std::fprintf(f, "%% %s\n", comment);
    std::fprintf(f, "%d %d %d\n", rows, cols, nnz);
    for (int32_t i = 0; i < rows; ++i)
        for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
            std::fprintf(f, "%d %d %.15e\n", i + 1, col_idx[k] + 1, values[k]);
    std::fclose(f);
    return HAMLSS_OK;
}

// Parse a MatrixMarket matrix and upload it (hamlss_mat_upload on the parsed CSR).
int hamlss_mat_load_mtx(hamlss_ctx* ctx, const char* path, hamlss_mat** out) {
    if (!ctx || !path || !out) return fail(HAMLSS_ERR_INVALID, "null argument");
    CsrHost A;
    int rc = load_csr(path, &A);
    if (rc) return rc;
    return hamlss_mat_upload(ctx, A.rows, A.cols, (int32_t)A.ci.size(), A.rp.data(), A.ci.data(), A.v.data(),
                             HAMLSS_HOST, out);
}

}  // extern "C"
