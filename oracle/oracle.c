/*
 * oracle.c -- CPU restatement of the HAMLSS solve path.  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this file's
 * library, and only as the checker; the device engine never calls it.
 *
 * Each function follows one reference function (cited file:line in the reference
 * project).  Floating-point expressions keep the reference's operation order, and the
 * library is compiled with -ffp-contract=off so that no multiply-add is fused: that is
 * what the reference's own sources give when built without -march=native / -ffast-math.
 * Reductions are sequential in index order (the reference at OMP_NUM_THREADS=1).
 *
 * Pinned against the reference built from its sources (tests/test_oracle_pin.py) and
 * against the fixtures in tests/golden/.
 */
#define _POSIX_C_SOURCE 199309L
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define REAL_EPS DBL_EPSILON

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }

/* ======================================================================= generators */

/* SparseMatrix::poisson_2d (sparse_matrix.cpp:288-311) after from_coo's (row,col) sort
 * (:242-282): row i*n+j holds (i-1,j) (i,j-1) (i,j) (i,j+1) (i+1,j) in column order. */
int64_t orc_poisson_2d(int32_t n, int32_t* rp, int32_t* ci, double* v) {
    int64_t k = 0;
    rp[0] = 0;
    for (int32_t i = 0; i < n; ++i)
        for (int32_t j = 0; j < n; ++j) {
            int32_t row = i * n + j;
            if (i > 0)     { ci[k] = row - n; v[k] = -1.0; ++k; }
            if (j > 0)     { ci[k] = row - 1; v[k] = -1.0; ++k; }
            ci[k] = row; v[k] = 4.0; ++k;
            if (j < n - 1) { ci[k] = row + 1; v[k] = -1.0; ++k; }
            if (i < n - 1) { ci[k] = row + n; v[k] = -1.0; ++k; }
            rp[row + 1] = (int32_t)k;
        }
    return k;
}

/* SparseMatrix::convection_diffusion_2d (sparse_matrix.cpp:317-350).  The diagonal is
 * accumulated in the reference's push order (west, east, north, south); entries are
 * then emitted in column order as from_coo sorts them. */
int64_t orc_convdiff_2d(int32_t n, double eps, double bx, double by,
                        int32_t* rp, int32_t* ci, double* v) {
    const double h = 1.0 / (n + 1);
    const double eh = eps / (h * h);
    const double bxh = bx / (2.0 * h);
    const double byh = by / (2.0 * h);
    int64_t k = 0;
    rp[0] = 0;
    for (int32_t i = 0; i < n; ++i)
        for (int32_t j = 0; j < n; ++j) {
            int32_t row = i * n + j;
            double diag = 4.0 * eh;
            double w = 0, e = 0, no = 0, so = 0;
            if (j > 0)     { w  = -eh + dmax(bxh, 0.0);  diag += dmax(-bxh, 0.0); }
            if (j < n - 1) { e  = -eh - dmin(bxh, 0.0);  diag += dmax(bxh, 0.0); }
            if (i > 0)     { no = -eh + dmax(byh, 0.0);  diag += dmax(-byh, 0.0); }
            if (i < n - 1) { so = -eh - dmin(byh, 0.0);  diag += dmax(byh, 0.0); }
            if (i > 0)     { ci[k] = row - n; v[k] = no; ++k; }
            if (j > 0)     { ci[k] = row - 1; v[k] = w;  ++k; }
            ci[k] = row; v[k] = diag; ++k;
            if (j < n - 1) { ci[k] = row + 1; v[k] = e;  ++k; }
            if (i < n - 1) { ci[k] = row + n; v[k] = so; ++k; }
            rp[row + 1] = (int32_t)k;
        }
    return k;
}

/* ========================================================================== kernels */

/* SparseMatrix::spmv (sparse_matrix.cpp:68-87). */
void orc_spmv(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
              const double* x, double* y) {
    for (int32_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
        y[i] = s;
    }
}

/* Vector::dot (vector.cpp:39-49), sequential. */
double orc_dot(int32_t n, const double* a, const double* b) {
    double s = 0.0;
    for (int32_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

static double orc_norm2(int32_t n, const double* a) { return sqrt(orc_dot(n, a, a)); }

/* =========================================================================== Jacobi */

/* JacobiPreconditioner::setup (jacobi.cpp:13-38). */
int orc_jacobi_setup(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                     double omega, double* inv_diag) {
    for (int32_t i = 0; i < n; ++i) {
        double d = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) { d = v[k]; break; }
        if (fabs(d) < REAL_EPS) return HAMLSS_ERR_ZERO_DIAG;
        inv_diag[i] = omega / d;
    }
    return HAMLSS_OK;
}

/* ============================================================================ ILU(0) */

/* ILUPreconditioner::setup_ilu0 (ilu.cpp:41-89): in-place IKJ on the pattern of A. */
int orc_ilu0_factor(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                    double* lu) {
    memcpy(lu, v, sizeof(double) * (size_t)rp[n]);
    int32_t* pos = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i) pos[i] = -1;
    int rc = HAMLSS_OK;
    for (int32_t i = 1; i < n && rc == HAMLSS_OK; ++i) {
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) pos[ci[p]] = p;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            int32_t k = ci[p];
            if (k >= i) break;
            double dk = 0.0;
            for (int32_t q = rp[k]; q < rp[k + 1]; ++q)
                if (ci[q] == k) { dk = lu[q]; break; }
            if (fabs(dk) < REAL_EPS) { rc = HAMLSS_ERR_ZERO_PIVOT; break; }
            lu[p] /= dk;
            double lik = lu[p];
            for (int32_t q = rp[k]; q < rp[k + 1]; ++q) {
                int32_t j = ci[q];
                if (j <= k) continue;
                int32_t pij = pos[j];
                if (pij < 0) continue;
                lu[pij] -= lik * lu[q];
            }
        }
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) pos[ci[p]] = -1;
    }
    free(pos);
    return rc;
}

/* ===================================================================== ILUT(tau, p) */

static int cmp_i32(const void* a, const void* b);

typedef struct { int32_t col; double val; } ilut_entry;

/* keep_largest (ilu.cpp:186-197): std::partial_sort by |value| (descending), i.e. a heap
 * select over the row in column order -- a heap of the first `keep` entries whose top is
 * the smallest magnitude, replaced by every later entry of strictly larger magnitude --
 * then the kept entries sorted by column.  The heap operations are the standard ones:
 * sift the hole down to a leaf along the child that comes first, then push the value
 * back up (the library's make_heap / pop_heap). */
static int ilut_first(const ilut_entry* a, const ilut_entry* b) {   /* comp(a, b) */
    return fabs(a->val) > fabs(b->val);
}

static void ilut_adjust(ilut_entry* h, long hole, long len, ilut_entry value) {
    const long top = hole;
    long child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (ilut_first(&h[child], &h[child - 1])) --child;
        h[hole] = h[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        h[hole] = h[child - 1];
        hole = child - 1;
    }
    long parent = (hole - 1) / 2;
    while (hole > top && ilut_first(&h[parent], &value)) {
        h[hole] = h[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    h[hole] = value;
}

static int ilut_by_col(const void* a, const void* b) {
    const ilut_entry* x = (const ilut_entry*)a;
    const ilut_entry* y = (const ilut_entry*)b;
    return (x->col > y->col) - (x->col < y->col);
}

static void ilut_keep_largest(ilut_entry* row, int32_t* len, int32_t keep) {
    if (keep <= 0 || *len <= keep) return;
    for (long parent = (keep - 2) / 2; keep >= 2; --parent) {          /* make_heap */
        ilut_adjust(row, parent, keep, row[parent]);
        if (parent == 0) break;
    }
    for (int32_t i = keep; i < *len; ++i) {                           /* heap select */
        if (ilut_first(&row[i], &row[0])) {
            ilut_entry v = row[i];
            row[i] = row[0];
            ilut_adjust(row, 0, keep, v);
        }
    }
    *len = keep;
    qsort(row, (size_t)keep, sizeof(ilut_entry), ilut_by_col);
}

/* ILUPreconditioner::setup_ilut (ilu.cpp:94-220): row-by-row threshold factorisation with
 * a dense work row.  The reference scans every k < i and every column to collect the row;
 * here the work row's touched columns are kept in a list and the pending pivots in a min
 * heap, which visits the same columns in the same (ascending) order.  Output: the L\U
 * rows (L entries, then the diagonal and U entries, each in column order).  Call with
 * out_ci == NULL to learn the entry count. */
int orc_ilut_factor(int32_t n, const int32_t* rp, const int32_t* ci, const double* v, double drop_tol,
                    int32_t fill_p, int32_t* out_rp, int32_t* out_ci, double* out_lu, int64_t* nnz_out) {
    double* w = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    unsigned char* active = (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1);
    unsigned char* touched = (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1);
    int32_t* tlist = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* heap = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* Lstart = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    int32_t* Ustart = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    size_t cap = (size_t)(rp[n] > 0 ? rp[n] : 1) * 2 + 16, used = 0;
    ilut_entry* store = (ilut_entry*)malloc(sizeof(ilut_entry) * cap);
    ilut_entry* rowbuf = (ilut_entry*)malloc(sizeof(ilut_entry) * (size_t)(n > 0 ? n : 1));
    int32_t* ulen = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* llen = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i) {
        int32_t nt = 0, nh = 0;
        double row_norm = 0.0;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int32_t j = ci[p];
            w[j] = v[p];
            active[j] = 1;
            if (!touched[j]) { touched[j] = 1; tlist[nt++] = j; }
            row_norm += v[p] * v[p];
        }
        row_norm = sqrt(row_norm);
        const double tau = drop_tol * row_norm;
        /* pending pivots: active columns < i, smallest first (binary min-heap) */
#define HEAP_PUSH(x) do { int32_t c_ = nh++; heap[c_] = (x); \
            while (c_ > 0 && heap[(c_ - 1) / 2] > heap[c_]) { int32_t t_ = heap[c_]; \
                heap[c_] = heap[(c_ - 1) / 2]; heap[(c_ - 1) / 2] = t_; c_ = (c_ - 1) / 2; } } while (0)
        for (int32_t t = 0; t < nt; ++t) if (tlist[t] < i) HEAP_PUSH(tlist[t]);
        while (nh > 0) {
            const int32_t k = heap[0];
            heap[0] = heap[--nh];
            for (int32_t c = 0;;) {
                int32_t l = 2 * c + 1, r = l + 1, m = c;
                if (l < nh && heap[l] < heap[m]) m = l;
                if (r < nh && heap[r] < heap[m]) m = r;
                if (m == c) break;
                int32_t t = heap[c]; heap[c] = heap[m]; heap[m] = t; c = m;
            }
            if (!active[k]) continue;
            if (fabs(w[k]) < tau) { w[k] = 0.0; active[k] = 0; continue; }
            double ukk = 0.0;
            const ilut_entry* U = store + Ustart[k];
            for (int32_t q = 0; q < ulen[k]; ++q)
                if (U[q].col == k) { ukk = U[q].val; break; }
            if (fabs(ukk) < REAL_EPS) { active[k] = 0; continue; }
            const double lik = w[k] / ukk;
            w[k] = lik;
            for (int32_t q = 0; q < ulen[k]; ++q) {
                const int32_t j = U[q].col;
                if (j <= k) continue;
                const double prod = lik * U[q].val;
                if (!touched[j]) { touched[j] = 1; tlist[nt++] = j; }
                if (!active[j] && fabs(prod) >= tau) {
                    active[j] = 1;
                    if (j < i) HEAP_PUSH(j);
                }
                w[j] -= prod;
            }
        }
#undef HEAP_PUSH
        /* collect L (j < i), the diagonal, U (j > i) in column order */
        qsort(tlist, (size_t)nt, sizeof(int32_t), cmp_i32);
        int32_t nl = 0, nu = 0;
        ilut_entry* Lrow = rowbuf;
        for (int32_t t = 0; t < nt && tlist[t] < i; ++t) {
            const int32_t j = tlist[t];
            if (active[j] && fabs(w[j]) >= tau) { Lrow[nl].col = j; Lrow[nl].val = w[j]; ++nl; }
        }
        const int32_t orig = rp[i + 1] - rp[i];
        ilut_keep_largest(Lrow, &nl, orig + fill_p);
        if (used + (size_t)nl + (size_t)nt + 1 > cap) {
            while (used + (size_t)nl + (size_t)nt + 1 > cap) cap *= 2;
            store = (ilut_entry*)realloc(store, sizeof(ilut_entry) * cap);
        }
        Lstart[i] = (int32_t)used;
        memcpy(store + used, Lrow, sizeof(ilut_entry) * (size_t)nl);
        used += (size_t)nl;
        llen[i] = nl;
        ilut_entry* Urow = rowbuf;
        double diag = w[i];
        if (fabs(diag) < REAL_EPS) diag = (diag >= 0 ? 1.0 : -1.0) * REAL_EPS * 1e6;
        Urow[nu].col = i; Urow[nu].val = diag; ++nu;
        for (int32_t t = 0; t < nt; ++t) {
            const int32_t j = tlist[t];
            if (j <= i) continue;
            if (active[j] && fabs(w[j]) >= tau) { Urow[nu].col = j; Urow[nu].val = w[j]; ++nu; }
        }
        ilut_keep_largest(Urow, &nu, orig + fill_p);
        Ustart[i] = (int32_t)used;
        memcpy(store + used, Urow, sizeof(ilut_entry) * (size_t)nu);
        used += (size_t)nu;
        ulen[i] = nu;
        for (int32_t t = 0; t < nt; ++t) {
            const int32_t j = tlist[t];
            w[j] = 0.0; active[j] = 0; touched[j] = 0;
        }
    }
    *nnz_out = (int64_t)used;
    if (out_ci) {
        int64_t pos = 0;
        out_rp[0] = 0;
        for (int32_t i = 0; i < n; ++i) {
            for (int32_t q = 0; q < llen[i]; ++q) { out_ci[pos] = store[Lstart[i] + q].col; out_lu[pos] = store[Lstart[i] + q].val; ++pos; }
            for (int32_t q = 0; q < ulen[i]; ++q) { out_ci[pos] = store[Ustart[i] + q].col; out_lu[pos] = store[Ustart[i] + q].val; ++pos; }
            out_rp[i + 1] = (int32_t)pos;
        }
    }
    free(w); free(active); free(touched); free(tlist); free(heap); free(Lstart); free(Ustart);
    free(store); free(rowbuf); free(ulen); free(llen);
    return HAMLSS_OK;
}

/* forward_sub / backward_sub / apply (ilu.cpp:225-271). */
int orc_ilu_apply(int32_t n, const int32_t* rp, const int32_t* ci, const double* lu,
                  const double* r, double* z) {
    double* y = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i) {
        double s = r[i];
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            int32_t j = ci[p];
            if (j >= i) break;
            s -= lu[p] * y[j];
        }
        y[i] = s;
    }
    int rc = HAMLSS_OK;
    for (int32_t i = n - 1; i >= 0; --i) {
        double s = y[i], d = 1.0;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            int32_t j = ci[p];
            if (j == i) { d = lu[p]; continue; }
            if (j > i) s -= lu[p] * z[j];
        }
        if (fabs(d) < REAL_EPS) { rc = HAMLSS_ERR_ZERO_PIVOT; break; }
        z[i] = s / d;
    }
    free(y);
    return rc;
}

/* Level sets of the triangular sweeps.  No reference counterpart (the reference sweeps
 * sequentially, ilu.cpp:225-262); the definition is the dependency depth of each row. */
int32_t orc_levels(int32_t n, const int32_t* rp, const int32_t* ci, int which, int32_t* level) {
    int32_t nlev = 0;
    if (which == 0) {
        for (int32_t i = 0; i < n; ++i) {
            int32_t l = 0;
            for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
                int32_t j = ci[p];
                if (j < i && level[j] + 1 > l) l = level[j] + 1;
            }
            level[i] = l;
            if (l + 1 > nlev) nlev = l + 1;
        }
    } else {
        for (int32_t i = n - 1; i >= 0; --i) {
            int32_t l = 0;
            for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
                int32_t j = ci[p];
                if (j > i && level[j] + 1 > l) l = level[j] + 1;
            }
            level[i] = l;
            if (l + 1 > nlev) nlev = l + 1;
        }
    }
    return nlev;
}

/* ============================================================================ SA-AMG */

typedef struct { int32_t rows, cols, nnz; int32_t* rp; int32_t* ci; double* v; } csr_t;

static void csr_free(csr_t* a) { free(a->rp); free(a->ci); free(a->v); memset(a, 0, sizeof(*a)); }

static csr_t csr_copy(int32_t rows, int32_t cols, const int32_t* rp, const int32_t* ci,
                      const double* v) {
    csr_t a;
    a.rows = rows; a.cols = cols; a.nnz = rp[rows];
    a.rp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(rows + 1));
    a.ci = (int32_t*)malloc(sizeof(int32_t) * (size_t)(a.nnz > 0 ? a.nnz : 1));
    a.v  = (double*)malloc(sizeof(double) * (size_t)(a.nnz > 0 ? a.nnz : 1));
    memcpy(a.rp, rp, sizeof(int32_t) * (size_t)(rows + 1));
    if (a.nnz) { memcpy(a.ci, ci, sizeof(int32_t) * (size_t)a.nnz); memcpy(a.v, v, sizeof(double) * (size_t)a.nnz); }
    return a;
}

/* AMGPreconditioner::aggregate (amg.cpp:30-67). */
int32_t orc_amg_aggregate(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                          double theta, int32_t* agg) {
    double* rmax = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int32_t i = 0; i < n; ++i) {
        agg[i] = -1;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] != i) rmax[i] = dmax(rmax[i], fabs(v[k]));
    }
    int32_t nagg = 0;
    for (int32_t i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        agg[i] = nagg;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            int32_t j = ci[k];
            if (j == i || agg[j] >= 0) continue;
            if (fabs(v[k]) >= theta * rmax[i]) agg[j] = nagg;
        }
        ++nagg;
    }
    for (int32_t i = 0; i < n; ++i)
        if (agg[i] < 0) agg[i] = nagg++;
    free(rmax);
    return nagg;
}

/* smooth_prolongation_op (amg.cpp:101-178) with one sweep on the tentative P of
 * build_prolongation (:73-89), computed sparsely.  Row i of the dense buffer starts as
 * e_{agg[i]}; each off-diagonal a_ij (in row order) subtracts (id*a_ij)*P_raw[j,c], which
 * is exactly id*a_ij at c = agg[j] and a signed zero elsewhere, so accumulating only at
 * c = agg[j] in the same order gives the dense result bit for bit.  Entries with
 * |v| <= 1e-14 are dropped (:160-176). */
static csr_t smooth_prolongation(const csr_t* A, const int32_t* agg, int32_t nc, double omega) {
    const int32_t n = A->rows;
    csr_t P;
    P.rows = n; P.cols = nc;
    P.rp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    size_t cap = (size_t)A->nnz + 1;
    P.ci = (int32_t*)malloc(sizeof(int32_t) * cap);
    P.v  = (double*)malloc(sizeof(double) * cap);
    int32_t* cols = (int32_t*)malloc(sizeof(int32_t) * 64);
    double* vals = (double*)malloc(sizeof(double) * 64);
    int32_t ccap = 64;
    int64_t k = 0;
    P.rp[0] = 0;
    for (int32_t i = 0; i < n; ++i) {
        int32_t m = 0;
        int32_t rl = A->rp[i + 1] - A->rp[i] + 1;
        if (rl > ccap) {
            ccap = rl;
            cols = (int32_t*)realloc(cols, sizeof(int32_t) * (size_t)ccap);
            vals = (double*)realloc(vals, sizeof(double) * (size_t)ccap);
        }
        cols[m] = agg[i]; vals[m] = 1.0; ++m;
        double id = 0.0;
        for (int32_t a = A->rp[i]; a < A->rp[i + 1]; ++a)
            if (A->ci[a] == i) { id = (fabs(A->v[a]) > REAL_EPS) ? omega / A->v[a] : 0.0; break; }
        if (!(fabs(id) < REAL_EPS)) {
            for (int32_t a = A->rp[i]; a < A->rp[i + 1]; ++a) {
                int32_t j = A->ci[a];
                if (j == i) continue;
                int32_t c = agg[j];
                double t = id * A->v[a] * 1.0;
                int32_t s = 0;
                while (s < m && cols[s] != c) ++s;
                if (s == m) { cols[m] = c; vals[m] = 0.0; ++m; }
                vals[s] -= t;
            }
        }
        /* emit in column order */
        for (int32_t a = 1; a < m; ++a) {           /* insertion sort, rows are short */
            int32_t cc = cols[a]; double vv = vals[a]; int32_t b = a - 1;
            while (b >= 0 && cols[b] > cc) { cols[b + 1] = cols[b]; vals[b + 1] = vals[b]; --b; }
            cols[b + 1] = cc; vals[b + 1] = vv;
        }
        for (int32_t a = 0; a < m; ++a)
            if (fabs(vals[a]) > 1e-14) { P.ci[k] = cols[a]; P.v[k] = vals[a]; ++k; }
        P.rp[i + 1] = (int32_t)k;
    }
    P.nnz = (int32_t)k;
    free(cols); free(vals);
    return P;
}

static csr_t tentative_prolongation(int32_t n, const int32_t* agg, int32_t nc) {
    csr_t P;
    P.rows = n; P.cols = nc; P.nnz = n;
    P.rp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    P.ci = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    P.v  = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i) { P.rp[i] = i; P.ci[i] = agg[i]; P.v[i] = 1.0; }
    P.rp[n] = n;
    return P;
}

/* transpose (sparse_matrix.cpp:138-165): counting sort, rows of A visited in order. */
static csr_t csr_transpose(const csr_t* A) {
    csr_t T;
    T.rows = A->cols; T.cols = A->rows; T.nnz = A->nnz;
    T.rp = (int32_t*)calloc((size_t)T.rows + 1, sizeof(int32_t));
    T.ci = (int32_t*)malloc(sizeof(int32_t) * (size_t)(T.nnz > 0 ? T.nnz : 1));
    T.v  = (double*)malloc(sizeof(double) * (size_t)(T.nnz > 0 ? T.nnz : 1));
    for (int32_t k = 0; k < A->nnz; ++k) T.rp[A->ci[k] + 1]++;
    for (int32_t j = 0; j < T.rows; ++j) T.rp[j + 1] += T.rp[j];
    int32_t* pos = (int32_t*)malloc(sizeof(int32_t) * (size_t)(T.rows > 0 ? T.rows : 1));
    for (int32_t j = 0; j < T.rows; ++j) pos[j] = T.rp[j];
    for (int32_t i = 0; i < A->rows; ++i)
        for (int32_t k = A->rp[i]; k < A->rp[i + 1]; ++k) {
            int32_t p = pos[A->ci[k]]++;
            T.ci[p] = i; T.v[p] = A->v[k];
        }
    free(pos);
    return T;
}

static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

/* mat_mat_product (sparse_matrix.cpp:171-237): per row, a dense accumulator summed in
 * (A entry, B entry) order; output columns sorted; |v| <= eps^2 dropped. */
static csr_t csr_spgemm(const csr_t* A, const csr_t* B) {
    const int32_t m = A->rows, n = B->cols;
    double* dense = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    char* flag = (char*)calloc((size_t)(n > 0 ? n : 1), 1);
    int32_t* touched = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    csr_t C;
    C.rows = m; C.cols = n;
    C.rp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m + 1));
    size_t cap = (size_t)A->nnz * 4 + 16;
    C.ci = (int32_t*)malloc(sizeof(int32_t) * cap);
    C.v  = (double*)malloc(sizeof(double) * cap);
    int64_t k = 0;
    C.rp[0] = 0;
    for (int32_t i = 0; i < m; ++i) {
        int32_t nt = 0;
        for (int32_t pa = A->rp[i]; pa < A->rp[i + 1]; ++pa) {
            int32_t j = A->ci[pa];
            double av = A->v[pa];
            for (int32_t pb = B->rp[j]; pb < B->rp[j + 1]; ++pb) {
                int32_t l = B->ci[pb];
                if (!flag[l]) { flag[l] = 1; touched[nt++] = l; }
                dense[l] += av * B->v[pb];
            }
        }
        qsort(touched, (size_t)nt, sizeof(int32_t), cmp_i32);
        if ((size_t)(k + nt) > cap) {
            while ((size_t)(k + nt) > cap) cap *= 2;
            C.ci = (int32_t*)realloc(C.ci, sizeof(int32_t) * cap);
            C.v  = (double*)realloc(C.v, sizeof(double) * cap);
        }
        for (int32_t t = 0; t < nt; ++t) {
            int32_t l = touched[t];
            if (fabs(dense[l]) > REAL_EPS * REAL_EPS) { C.ci[k] = l; C.v[k] = dense[l]; ++k; }
            dense[l] = 0.0; flag[l] = 0;
        }
        C.rp[i + 1] = (int32_t)k;
    }
    C.nnz = (int32_t)k;
    free(dense); free(flag); free(touched);
    return C;
}

typedef struct { csr_t A, P, R; double* dinv; } amg_level_t;

struct orc_amg {
    int32_t nlev;
    amg_level_t lev[32];
    double omega;
    int pre, post;
    /* coarsest dense LU is rebuilt on every V-cycle in the reference; kept identical */
};

static double* level_dinv(const csr_t* A) {
    double* d = (double*)malloc(sizeof(double) * (size_t)(A->rows > 0 ? A->rows : 1));
    for (int32_t i = 0; i < A->rows; ++i) {
        double di = 0.0;
        for (int32_t k = A->rp[i]; k < A->rp[i + 1]; ++k)
            if (A->ci[k] == i) { di = A->v[k]; break; }
        d[i] = (fabs(di) > REAL_EPS) ? 1.0 / di : 0.0;
    }
    return d;
}

/* AMGPreconditioner::setup (amg.cpp:183-237). */
orc_amg* orc_amg_setup(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                       const hamlss_params* p) {
    orc_amg* h = (orc_amg*)calloc(1, sizeof(orc_amg));
    h->omega = p->amg_omega;
    h->pre = p->amg_smooth_pre;
    h->post = p->amg_smooth_post;
    int32_t max_levels = p->amg_levels;
    int32_t coarse_limit = p->amg_coarse_limit;
    if (max_levels > 32) max_levels = 32;
    h->lev[0].A = csr_copy(n, n, rp, ci, v);
    h->lev[0].dinv = level_dinv(&h->lev[0].A);
    h->nlev = 1;
    for (int lv = 0; lv < max_levels - 1; ++lv) {
        csr_t* Af = &h->lev[h->nlev - 1].A;
        if (Af->rows <= coarse_limit) break;
        int32_t* agg = (int32_t*)malloc(sizeof(int32_t) * (size_t)Af->rows);
        int32_t nc = orc_amg_aggregate(Af->rows, Af->rp, Af->ci, Af->v, p->amg_strong, agg);
        if (nc >= Af->rows) { free(agg); break; }
        csr_t P = smooth_prolongation(Af, agg, nc, h->omega);
        free(agg);
        csr_t R = csr_transpose(&P);
        csr_t AP = csr_spgemm(Af, &P);
        csr_t Ac = csr_spgemm(&R, &AP);
        csr_free(&AP);
        h->lev[h->nlev - 1].P = P;
        h->lev[h->nlev - 1].R = R;
        h->lev[h->nlev].A = Ac;
        h->lev[h->nlev].dinv = level_dinv(&h->lev[h->nlev].A);
        h->nlev++;
    }
    return h;
}

void orc_amg_free(orc_amg* h) {
    if (!h) return;
    for (int l = 0; l < h->nlev; ++l) {
        csr_free(&h->lev[l].A); csr_free(&h->lev[l].P); csr_free(&h->lev[l].R);
        free(h->lev[l].dinv);
    }
    free(h);
}

int32_t orc_amg_num_levels(const orc_amg* h) { return h->nlev; }

int orc_amg_level(const orc_amg* h, int32_t level, int32_t which, int32_t* rows,
                  int32_t* cols, int32_t* nnz, int32_t* rp, int32_t* ci, double* v) {
    if (level < 0 || level >= h->nlev || which < 0 || which > 2) return HAMLSS_ERR_INVALID;
    const csr_t* a = which == 0 ? &h->lev[level].A : which == 1 ? &h->lev[level].P : &h->lev[level].R;
    if (!a->rp) return HAMLSS_ERR_INVALID;
    if (rows) *rows = a->rows;
    if (cols) *cols = a->cols;
    if (nnz) *nnz = a->nnz;
    if (rp) memcpy(rp, a->rp, sizeof(int32_t) * (size_t)(a->rows + 1));
    if (ci) memcpy(ci, a->ci, sizeof(int32_t) * (size_t)a->nnz);
    if (v) memcpy(v, a->v, sizeof(double) * (size_t)a->nnz);
    return HAMLSS_OK;
}

/* direct_solve (amg.cpp:260-291): dense Gaussian elimination with partial pivoting. */
static void dense_solve(const csr_t* A, const double* rhs, double* x) {
    const int32_t n = A->rows, w = n + 1;
    double* M = (double*)calloc((size_t)n * (size_t)w, sizeof(double));
    for (int32_t i = 0; i < n; ++i) {
        for (int32_t k = A->rp[i]; k < A->rp[i + 1]; ++k) M[(size_t)i * w + A->ci[k]] = A->v[k];
        M[(size_t)i * w + n] = rhs[i];
    }
    double* tmp = (double*)malloc(sizeof(double) * (size_t)w);
    for (int32_t col = 0; col < n; ++col) {
        int32_t piv = col;
        for (int32_t r = col + 1; r < n; ++r)
            if (fabs(M[(size_t)r * w + col]) > fabs(M[(size_t)piv * w + col])) piv = r;
        if (piv != col) {
            memcpy(tmp, &M[(size_t)col * w], sizeof(double) * (size_t)w);
            memcpy(&M[(size_t)col * w], &M[(size_t)piv * w], sizeof(double) * (size_t)w);
            memcpy(&M[(size_t)piv * w], tmp, sizeof(double) * (size_t)w);
        }
        if (fabs(M[(size_t)col * w + col]) < 1e-14) continue;
        double inv = 1.0 / M[(size_t)col * w + col];
        for (int32_t r = col + 1; r < n; ++r) {
            double f = M[(size_t)r * w + col] * inv;
            for (int32_t c = col; c <= n; ++c) M[(size_t)r * w + c] -= f * M[(size_t)col * w + c];
        }
    }
    for (int32_t i = n - 1; i >= 0; --i) {
        double s = M[(size_t)i * w + n];
        for (int32_t j = i + 1; j < n; ++j) s -= M[(size_t)i * w + j] * x[j];
        x[i] = (fabs(M[(size_t)i * w + i]) > 1e-14) ? s / M[(size_t)i * w + i] : 0.0;
    }
    free(tmp); free(M);
}

/* smooth (amg.cpp:242-254). */
static void amg_smooth(const orc_amg* h, int l, const double* rhs, double* x, int steps, double* res) {
    const csr_t* A = &h->lev[l].A;
    const double* dinv = h->lev[l].dinv;
    for (int s = 0; s < steps; ++s) {
        orc_spmv(A->rows, A->rp, A->ci, A->v, x, res);
        for (int32_t i = 0; i < A->rows; ++i) x[i] += h->omega * dinv[i] * (rhs[i] - res[i]);
    }
}

/* v_cycle (amg.cpp:296-335). */
static void amg_vcycle(const orc_amg* h, int l, const double* rhs, double* x) {
    if (l == h->nlev - 1) { dense_solve(&h->lev[l].A, rhs, x); return; }
    const csr_t* A = &h->lev[l].A;
    const csr_t* P = &h->lev[l].P;
    const csr_t* R = &h->lev[l].R;
    const int32_t n = A->rows, nc = R->rows;
    double* t = (double*)malloc(sizeof(double) * (size_t)n);
    double* res = (double*)malloc(sizeof(double) * (size_t)n);
    amg_smooth(h, l, rhs, x, h->pre, t);
    orc_spmv(n, A->rp, A->ci, A->v, x, t);
    for (int32_t i = 0; i < n; ++i) res[i] = rhs[i] - t[i];
    double* rc = (double*)malloc(sizeof(double) * (size_t)nc);
    double* ec = (double*)calloc((size_t)nc, sizeof(double));
    orc_spmv(nc, R->rp, R->ci, R->v, res, rc);
    amg_vcycle(h, l + 1, rc, ec);
    orc_spmv(n, P->rp, P->ci, P->v, ec, t);
    for (int32_t i = 0; i < n; ++i) x[i] += t[i];
    amg_smooth(h, l, rhs, x, h->post, t);
    free(t); free(res); free(rc); free(ec);
}

/* apply (amg.cpp:340-343). */
void orc_amg_apply(const orc_amg* h, const double* r, double* z) {
    memset(z, 0, sizeof(double) * (size_t)h->lev[0].A.rows);
    amg_vcycle(h, 0, r, z);
}

/* ========================================================== generic preconditioner */

struct orc_prec {
    int kind;
    int32_t n;
    const int32_t* rp;   /* pattern of A (caller keeps it alive), or of the ILUT factor */
    const int32_t* ci;
    double* data;        /* Jacobi inv_diag or ILU factor values */
    int32_t* frp;        /* ILUT: the factor's own pattern */
    int32_t* fci;
    orc_amg* amg;
};

orc_prec* orc_prec_setup(int kind, int32_t n, const int32_t* rp, const int32_t* ci,
                         const double* v, const hamlss_params* p, int* status) {
    *status = HAMLSS_OK;
    if (kind == HAMLSS_PREC_NONE) return NULL;
    orc_prec* M = (orc_prec*)calloc(1, sizeof(orc_prec));
    M->kind = kind; M->n = n; M->rp = rp; M->ci = ci;
    if (kind == HAMLSS_PREC_JACOBI) {
        M->data = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
        *status = orc_jacobi_setup(n, rp, ci, v, p->jacobi_omega, M->data);
    } else if (kind == HAMLSS_PREC_ILU) {
        /* SolverFactory::make_precond sets drop_tol only (solver_factory.cpp:73-77), so the
         * dispatch of ilu.cpp:31-36 picks ILUT exactly when drop_tol > 0, with fill 0 */
        if (p->drop_tol > 0.0) {
            int64_t nnz = 0;
            *status = orc_ilut_factor(n, rp, ci, v, p->drop_tol, 0, NULL, NULL, NULL, &nnz);
            if (*status == HAMLSS_OK) {
                M->frp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
                M->fci = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
                M->data = (double*)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
                *status = orc_ilut_factor(n, rp, ci, v, p->drop_tol, 0, M->frp, M->fci, M->data, &nnz);
                M->rp = M->frp;
                M->ci = M->fci;
            }
        } else {
            M->data = (double*)malloc(sizeof(double) * (size_t)(rp[n] > 0 ? rp[n] : 1));
            *status = orc_ilu0_factor(n, rp, ci, v, M->data);
        }
    } else if (kind == HAMLSS_PREC_AMG) {
        M->amg = orc_amg_setup(n, rp, ci, v, p);
    } else {
        *status = HAMLSS_ERR_INVALID;
    }
    if (*status != HAMLSS_OK) { orc_prec_free(M); return NULL; }
    return M;
}

void orc_prec_free(orc_prec* M) {
    if (!M) return;
    free(M->data);
    free(M->frp);
    free(M->fci);
    orc_amg_free(M->amg);
    free(M);
}

int orc_prec_apply(const orc_prec* M, const double* r, double* z) {
    if (M->kind == HAMLSS_PREC_JACOBI) {
        for (int32_t i = 0; i < M->n; ++i) z[i] = M->data[i] * r[i];
        return HAMLSS_OK;
    }
    if (M->kind == HAMLSS_PREC_ILU) return orc_ilu_apply(M->n, M->rp, M->ci, M->data, r, z);
    if (M->kind == HAMLSS_PREC_AMG) { orc_amg_apply(M->amg, r, z); return HAMLSS_OK; }
    return HAMLSS_ERR_INVALID;
}

static void precond(const orc_prec* M, int32_t n, const double* r, double* z, int* rc) {
    if (M) { int s = orc_prec_apply(M, r, z); if (s != HAMLSS_OK) *rc = s; }
    else memcpy(z, r, sizeof(double) * (size_t)n);
}

/* ================================================================================ CG */

/* flop_model (energy_monitor.hpp:163-177) */
static int64_t spmv_flops(int32_t nz) { return 2LL * nz; }
static int64_t spmv_bytes(int32_t n, int32_t nz) { return (int64_t)(n + 1 + nz) * 4 + (int64_t)nz * 8 + (int64_t)n * 16; }

/* CGSolver::solve (cg_solver.cpp:37-191). */
int orc_cg(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
           const orc_prec* M, const double* b, double* x, const hamlss_params* p,
           hamlss_stats* st) {
    double t0 = now_s();
    const int32_t nz = rp[n];
    const double tol = p->tol;
    int rc = HAMLSS_OK;
    size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double *r = (double*)malloc(sz), *z = (double*)malloc(sz), *pp = (double*)malloc(sz),
           *q = (double*)malloc(sz);
    orc_spmv(n, rp, ci, v, x, r);
    for (int32_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
    const double bn = orc_norm2(n, b);
    const double r0 = orc_norm2(n, r);
    st->initial_residual = r0;
    if (bn < REAL_EPS) {
        st->converged = 1; st->final_residual = r0; st->iterations = 0;
        free(r); free(z); free(pp); free(q);
        return 1;
    }
    double rel = r0 / bn;
    if (rel < tol) {
        st->converged = 1; st->final_residual = rel; st->iterations = 0;
        free(r); free(z); free(pp); free(q);
        return 1;
    }
    precond(M, n, r, z, &rc);
    memcpy(pp, z, sz);
    double rho = orc_dot(n, r, z), rho_old = rho;
    st->solver_used = HAMLSS_SOLVER_CG;
    st->precond_used = M ? M->kind : HAMLSS_PREC_NONE;
    int64_t flops = 0, bytes = 0;
    int iter = 0;
    for (; iter < p->max_iter && rc == HAMLSS_OK; ++iter) {
        orc_spmv(n, rp, ci, v, pp, q);
        flops += spmv_flops(nz); bytes += spmv_bytes(n, nz);
        double pq = orc_dot(n, pp, q);
        flops += 2LL * n; bytes += 16LL * n;
        if (fabs(pq) < REAL_EPS * 1e6 * fabs(rho)) {
            orc_spmv(n, rp, ci, v, x, pp);
            for (int32_t i = 0; i < n; ++i) r[i] = b[i] - pp[i];
            precond(M, n, r, z, &rc);
            memcpy(pp, z, sz);
            rho = orc_dot(n, r, z);
            st->restarts++;
            continue;
        }
        double alpha = rho / pq;
        for (int32_t i = 0; i < n; ++i) x[i] += alpha * pp[i];
        flops += 2LL * n; bytes += 24LL * n;
        for (int32_t i = 0; i < n; ++i) r[i] += -alpha * q[i];
        flops += 2LL * n; bytes += 24LL * n;
        rel = orc_norm2(n, r) / bn;
        if (rel < tol) { ++iter; break; }
        precond(M, n, r, z, &rc);
        rho_old = rho;
        rho = orc_dot(n, r, z);
        flops += 2LL * n; bytes += 16LL * n;
        if (fabs(rho_old) < REAL_EPS * 1e8 * fabs(rho)) {
            orc_spmv(n, rp, ci, v, x, z);
            for (int32_t i = 0; i < n; ++i) r[i] = b[i] - z[i];
            precond(M, n, r, z, &rc);
            memcpy(pp, z, sz);
            rho = orc_dot(n, r, z);
            rho_old = rho;
            st->restarts++;
            continue;
        }
        double beta = rho / rho_old;
        for (int32_t i = 0; i < n; ++i) pp[i] = 1.0 * z[i] + beta * pp[i];
        flops += 2LL * n; bytes += 24LL * n;
    }
    st->iterations = iter;
    st->final_residual = rel;
    st->converged = rel < tol;
    st->solve_time_s = now_s() - t0;
    st->flop_count = flops;
    st->mem_bytes = bytes;
    st->energy_joules = 2.0e-10 * (double)flops + 5.0e-9 * (double)bytes;
    free(r); free(z); free(pp); free(q);
    if (rc != HAMLSS_OK) return rc;
    return st->converged;
}

/* ============================================================================ FGMRES */

/* compute_givens / apply_givens (fgmres_solver.cpp:36-51). */
static void givens(double f, double g, double* cs, double* sn, double* r) {
    if (fabs(g) < REAL_EPS) { *cs = 1.0; *sn = 0.0; *r = f; }
    else if (fabs(f) < REAL_EPS) { *cs = 0.0; *sn = 1.0; *r = g; }
    else { double t = sqrt(f * f + g * g); *cs = f / t; *sn = g / t; *r = t; }
}
static void rot(double* dx, double* dy, double cs, double sn) {
    double t = cs * *dx + sn * *dy;
    *dy = -sn * *dx + cs * *dy;
    *dx = t;
}

/* fgmres_cycle (fgmres_solver.cpp:72-160); H is (m+1) x m row-major. */
static int fgmres_cycle(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                        const orc_prec* M, const double* b, double* x, double tol_abs, int m,
                        double* res_norm, int* rc, int pipelined) {
    size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double* r = (double*)malloc(sz);
    orc_spmv(n, rp, ci, v, x, r);
    for (int32_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
    double beta = orc_norm2(n, r);
    *res_norm = beta;
    if (beta < tol_abs) { free(r); return 0; }
    double* V = (double*)calloc((size_t)(m + 1) * (size_t)(n > 0 ? n : 1), sizeof(double));
    double* Z = (double*)calloc((size_t)m * (size_t)(n > 0 ? n : 1), sizeof(double));
    double* w = (double*)malloc(sz);
    double* H = (double*)calloc((size_t)(m + 1) * (size_t)m, sizeof(double));
    double* cs = (double*)calloc((size_t)m, sizeof(double));
    double* sn = (double*)calloc((size_t)m, sizeof(double));
    double* g = (double*)calloc((size_t)m + 1, sizeof(double));
    memcpy(V, r, sz);
    double inv = 1.0 / beta;
    for (int32_t i = 0; i < n; ++i) V[i] *= inv;
    g[0] = beta;
#define HH(i, j) H[(size_t)(i) * (size_t)m + (size_t)(j)]
    int j = 0;
    for (; j < m; ++j) {
        double* vj = V + (size_t)j * n;
        double* zj = Z + (size_t)j * n;
        precond(M, n, vj, zj, rc);
        orc_spmv(n, rp, ci, v, zj, w);
        for (int i = 0; i <= j; ++i) {
            double* vi = V + (size_t)i * n;
            HH(i, j) = orc_dot(n, w, vi);
            double a = -HH(i, j);
            for (int32_t t = 0; t < n; ++t) w[t] += a * vi[t];
        }
        HH(j + 1, j) = orc_norm2(n, w);
        if (HH(j + 1, j) > REAL_EPS) {
            double* vn = V + (size_t)(j + 1) * n;
            double s = 1.0 / HH(j + 1, j);
            for (int32_t t = 0; t < n; ++t) vn[t] = w[t] * s;
        } else if (pipelined) {
            /* pipeline_cycle leaves on a lucky breakdown before rotating column j
             * (pipelined_fgmres_solver.cpp:117-123) */
            ++j;
            break;
        }
        for (int i = 0; i < j; ++i) rot(&HH(i, j), &HH(i + 1, j), cs[i], sn[i]);
        double rv;
        givens(HH(j, j), HH(j + 1, j), &cs[j], &sn[j], &rv);
        HH(j, j) = rv;
        HH(j + 1, j) = 0.0;
        rot(&g[j], &g[j + 1], cs[j], sn[j]);
        *res_norm = fabs(g[j + 1]);
        if (*res_norm < tol_abs) { ++j; break; }
    }
    /* solve_hessenberg (fgmres_solver.cpp:57-66) */
    double* y = (double*)calloc((size_t)(j > 0 ? j : 1), sizeof(double));
    for (int i = j - 1; i >= 0; --i) {
        double s = g[i];
        for (int k = i + 1; k < j; ++k) s -= HH(i, k) * y[k];
        y[i] = (fabs(HH(i, i)) > REAL_EPS) ? (s / HH(i, i)) : 0.0;
    }
#undef HH
    for (int i = 0; i < j; ++i) {
        const double* zi = Z + (size_t)i * n;
        for (int32_t t = 0; t < n; ++t) x[t] += y[i] * zi[t];
    }
    free(r); free(V); free(Z); free(w); free(H); free(cs); free(sn); free(g); free(y);
    return j;
}

/* FGMRESSolver::solve (fgmres_solver.cpp:165-241), or with pipelined = 1
 * PipelinedFGMRESSolver::solve (pipelined_fgmres_solver.cpp:168-242): the same Arnoldi
 * values (the pipelined cycle computes A M^-1 v_{j+1} one step early), its lucky-breakdown
 * exit, and its cost model of (steps + 1) SpMVs per cycle. */
static int fgmres_impl(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                       const orc_prec* M, const double* b, double* x, const hamlss_params* p,
                       hamlss_stats* st, int pipelined) {
    double t0 = now_s();
    const int32_t nz = rp[n];
    const int m = p->restart_size < n ? p->restart_size : n;
    int rc = HAMLSS_OK;
    const double bn = orc_norm2(n, b);
    if (bn < REAL_EPS) { st->converged = 1; st->final_residual = 0.0; return 1; }
    const double tol_abs = p->tol * bn;
    st->solver_used = HAMLSS_SOLVER_FGMRES;
    st->precond_used = M ? M->kind : HAMLSS_PREC_NONE;
    int64_t flops = 0, bytes = 0;
    double res = bn;
    int total = 0, restarts = 0;
    while (total < p->max_iter && rc == HAMLSS_OK) {
        int remaining = p->max_iter - total;
        int cm = m < remaining ? m : remaining;
        int it = fgmres_cycle(n, rp, ci, v, M, b, x, tol_abs, cm, &res, &rc, pipelined);
        const int64_t nspmv = it + (pipelined ? 1 : 0);
        flops += nspmv * spmv_flops(nz) + (int64_t)it * 4LL * n;
        bytes += nspmv * spmv_bytes(n, nz) + (int64_t)it * 32LL * n;
        total += it;
        ++restarts;
        double rel = res / bn;
        if (rel < p->tol || it == 0) { st->converged = rel < p->tol; st->final_residual = rel; break; }
    }
    st->iterations = total;
    st->restarts = restarts - 1;
    st->solve_time_s = now_s() - t0;
    st->flop_count = flops;
    st->mem_bytes = bytes;
    st->energy_joules = 2.0e-10 * (double)flops + 5.0e-9 * (double)bytes;
    if (rc != HAMLSS_OK) return rc;
    return st->converged;
}

int orc_fgmres(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
               const orc_prec* M, const double* b, double* x, const hamlss_params* p,
               hamlss_stats* st) {
    return fgmres_impl(n, rp, ci, v, M, b, x, p, st, 0);
}

int orc_pipelined_fgmres(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                         const orc_prec* M, const double* b, double* x, const hamlss_params* p,
                         hamlss_stats* st) {
    return fgmres_impl(n, rp, ci, v, M, b, x, p, st, 1);
}

/* ============================================================================ s-step */

/* SparseMatrix::spectral_interval (sparse_matrix.cpp:451-479). */
void orc_spectral_interval(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                           int steps, double* lo, double* hi) {
    const int K = n < steps ? n : steps;
    size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double *q = (double*)malloc(sz), *qp = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    double* Aq = (double*)malloc(sz);
    double alpha[64], beta[64];
    int na = 0, nb = 0;
    const double inv_sq_n = 1.0 / sqrt((double)n);
    for (int32_t i = 0; i < n; ++i) q[i] = inv_sq_n;
    double bj = 0.0;
    for (int j = 0; j < K && j < 64; ++j) {
        orc_spmv(n, rp, ci, v, q, Aq);
        const double aj = orc_dot(n, q, Aq);
        alpha[na++] = aj;
        for (int32_t i = 0; i < n; ++i) Aq[i] -= aj * q[i] + bj * qp[i];
        bj = orc_norm2(n, Aq);
        if (bj < REAL_EPS * 1e6) break;
        beta[nb++] = bj;
        memcpy(qp, q, sz);
        memcpy(q, Aq, sz);
        const double s = 1.0 / bj;
        for (int32_t i = 0; i < n; ++i) q[i] *= s;
    }
    double tmin = alpha[0], tmax = alpha[0];
    for (int i = 0; i < na; ++i) {
        double r = 0.0;
        if (i > 0) r += fabs(beta[i - 1]);
        if (i < na - 1) r += fabs(beta[i]);
        tmin = dmin(tmin, alpha[i] - r);
        tmax = dmax(tmax, alpha[i] + r);
    }
    *lo = tmin;
    *hi = tmax;
    free(q); free(qp); free(Aq);
}

/* build_basis (sstep_cg_solver.cpp:44-66) into B (k columns of n) and gram_matrix (:71-80). */
static void sstep_basis(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                        const double* r, double lam_min, double lam_max, int k, double* B,
                        double* tmp, double* G) {
    double shifts[64];
    const double c = 0.5 * (lam_min + lam_max), h = 0.5 * (lam_max - lam_min);
    for (int j = 0; j < k; ++j) shifts[j] = c + h * cos(3.14159265358979323846 * (2.0 * j + 1.0) / (2.0 * k));  /* M_PI */
    size_t sz = sizeof(double) * (size_t)n;
    memcpy(B, r, sz);
    const double n0 = orc_norm2(n, B);
    if (n0 > REAL_EPS) { const double s = 1.0 / n0; for (int32_t i = 0; i < n; ++i) B[i] *= s; }
    for (int j = 1; j < k; ++j) {
        double* prev = B + (size_t)(j - 1) * n;
        double* cur = B + (size_t)j * n;
        orc_spmv(n, rp, ci, v, prev, tmp);
        memcpy(cur, tmp, sz);
        const double a = -shifts[j - 1];
        for (int32_t i = 0; i < n; ++i) cur[i] += a * prev[i];
        const double nj = orc_norm2(n, cur);
        if (nj > REAL_EPS) { const double s = 1.0 / nj; for (int32_t i = 0; i < n; ++i) cur[i] *= s; }
    }
    for (int i = 0; i < k; ++i)
        for (int j = i; j < k; ++j) {
            G[i * k + j] = orc_dot(n, B + (size_t)i * n, B + (size_t)j * n);
            G[j * k + i] = G[i * k + j];
        }
}

/* SStepCGSolver::solve (sstep_cg_solver.cpp:170-305) with gram_condition_estimate
 * (:108-119) and local_lstsq (:125-164).  The preconditioner is not applied. */
int orc_sstep_cg(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                 const orc_prec* M, const double* b, double* x, const hamlss_params* p,
                 hamlss_stats* st) {
    double t0 = now_s();
    const int32_t nz = rp[n];
    if (p->sstep_k < 1 || p->sstep_k > 32) return HAMLSS_ERR_INVALID;
    int k = p->sstep_k;
    const int kcap = n / 10 > 1 ? n / 10 : 1;
    if (kcap < k) k = kcap;
    double lo, hi;
    orc_spectral_interval(n, rp, ci, v, 20, &lo, &hi);
    const double lam_min = dmax(lo, REAL_EPS);
    const double lam_max = dmax(hi, lam_min * 2.0);
    size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double* r = (double*)malloc(sz);
    orc_spmv(n, rp, ci, v, x, r);
    for (int32_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
    const double bn = orc_norm2(n, b);
    double rn = orc_norm2(n, r);
    st->initial_residual = rn;
    if (bn < REAL_EPS) { st->converged = 1; st->final_residual = 0.0; free(r); return 1; }
    double rel = rn / bn;
    if (rel < p->tol) { st->converged = 1; st->final_residual = rel; free(r); return 1; }
    st->solver_used = HAMLSS_SOLVER_SSTEP_CG;
    st->precond_used = M ? M->kind : HAMLSS_PREC_NONE;
    st->sstep_k = k;
    double* B = (double*)malloc(sz * (size_t)k);
    double* tmp = (double*)malloc(sz);
    double* Ap = (double*)malloc(sz);
    double G[32 * 32], L[32 * 32], rhs[32], z[32], y[32];
    int64_t flops = 0, bytes = 0;
    int total = 0;
    while (total < p->max_iter && rel > p->tol) {
        int kb = k;
        sstep_basis(n, rp, ci, v, r, lam_min, lam_max, kb, B, tmp, G);
        flops += (int64_t)kb * spmv_flops(nz);
        bytes += (int64_t)kb * spmv_bytes(n, nz);
        double mx = 0.0, mn = INFINITY;
        for (int i = 0; i < kb; ++i) {
            const double d = fabs(G[i * kb + i]);
            mx = dmax(mx, d);
            if (d > REAL_EPS) mn = dmin(mn, d);
        }
        const double cond = (mn >= mx) ? 1.0 : mx / mn;
        if (cond > p->sstep_cond_tol && kb > 1) {
            kb = kb / 2 > 1 ? kb / 2 : 1;
            sstep_basis(n, rp, ci, v, r, lam_min, lam_max, kb, B, tmp, G);
        }
        st->comm_bytes += 1;
        for (int i = 0; i < kb; ++i) rhs[i] = orc_dot(n, r, B + (size_t)i * n);
        flops += (int64_t)kb * 2LL * n;
        int ok = 1;
        for (int i = 0; i < kb && ok; ++i)
            for (int j = 0; j <= i; ++j) {
                double s = G[i * kb + j];
                for (int l = 0; l < j; ++l) s -= L[i * kb + l] * L[j * kb + l];
                if (i == j) {
                    if (s <= 0.0) { ok = 0; break; }
                    L[i * kb + j] = sqrt(s);
                } else {
                    L[i * kb + j] = s / L[j * kb + j];
                }
            }
        if (!ok) {
            /* one steepest-descent step (:236-250) */
            orc_spmv(n, rp, ci, v, r, Ap);
            const double rr = orc_dot(n, r, r), rAp = orc_dot(n, r, Ap);
            if (fabs(rAp) > REAL_EPS) {
                const double alpha = rr / rAp;
                for (int32_t i = 0; i < n; ++i) x[i] += alpha * r[i];
                for (int32_t i = 0; i < n; ++i) r[i] += -alpha * Ap[i];
            }
            ++total;
            rel = orc_norm2(n, r) / bn;
            continue;
        }
        for (int i = 0; i < kb; ++i) {
            double s = rhs[i];
            for (int j = 0; j < i; ++j) s -= L[i * kb + j] * z[j];
            z[i] = s / L[i * kb + i];
        }
        for (int i = kb - 1; i >= 0; --i) {
            double s = z[i];
            for (int j = i + 1; j < kb; ++j) s -= L[j * kb + i] * y[j];
            y[i] = s / L[i * kb + i];
        }
        for (int i = 0; i < kb; ++i) {
            const double* Bi = B + (size_t)i * n;
            for (int32_t t = 0; t < n; ++t) x[t] += y[i] * Bi[t];
        }
        orc_spmv(n, rp, ci, v, x, r);
        flops += spmv_flops(nz);
        bytes += spmv_bytes(n, nz);
        for (int32_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
        rn = orc_norm2(n, r);
        rel = rn / bn;
        total += kb;
    }
    st->iterations = total;
    st->final_residual = rel;
    st->converged = rel < p->tol;
    st->solve_time_s = now_s() - t0;
    st->flop_count = flops;
    st->mem_bytes = bytes;
    st->energy_joules = 2e-10 * (double)flops + 5e-9 * (double)bytes;
    free(r); free(B); free(tmp); free(Ap);
    return st->converged;
}

/* ========================================================================= adaptive */

static int32_t find_entry(const int32_t* rp, const int32_t* ci, int32_t i, int32_t j) {
    int32_t lo = rp[i], hi = rp[i + 1];
    while (lo < hi) { int32_t mid = lo + (hi - lo) / 2; if (ci[mid] < j) lo = mid + 1; else hi = mid; }
    return (lo < rp[i + 1] && ci[lo] == j) ? lo : -1;
}
static double get_entry(const int32_t* rp, const int32_t* ci, const double* v, int32_t i, int32_t j) {
    int32_t k = find_entry(rp, ci, i, j);
    return k >= 0 ? v[k] : 0.0;
}

/* AdaptiveSelector::extract_features + select_initial_state (adaptive_selector.cpp:37-233),
 * with the SparseMatrix helpers of sparse_matrix.cpp:355-493.  feat[] is the order of
 * MatrixFeatures::to_feature_vector (:418-446). */
int orc_extract_features(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                         double feat[24], int32_t* initial_state) {
    const int32_t nnz = rp[n];
    double density = (n == 0) ? 0.0 : (double)nnz / ((double)n * n);
    double fro = 0.0;
    for (int32_t k = 0; k < nnz; ++k) fro += v[k] * v[k];
    fro = sqrt(fro);
    double min_dd = INFINITY;
    for (int32_t i = 0; i < n; ++i) {
        double da = 0.0, off = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            if (ci[k] == i) da = fabs(v[k]); else off += fabs(v[k]);
        }
        double dd = (off > REAL_EPS) ? (da / off) : INFINITY;
        if (dd < min_dd) min_dd = dd;
    }
    double diag_dom = (min_dd == INFINITY) ? 1.0 : min_dd;
    /* Lanczos-30 + Gershgorin (:66-126) */
    double cond, lam_max, lam_min;
    {
        int K = n < 30 ? n : 30;
        double inv_sqrt_n = 1.0 / sqrt((double)n);
        size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
        double *q = (double*)malloc(sz), *qp = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double)),
               *Aq = (double*)malloc(sz);
        for (int32_t i = 0; i < n; ++i) q[i] = inv_sqrt_n;
        double al[30], be[30];
        int na = 0, nb = 0;
        double bj = 0.0;
        for (int j = 0; j < K; ++j) {
            orc_spmv(n, rp, ci, v, q, Aq);
            double aj = orc_dot(n, q, Aq);
            al[na++] = aj;
            for (int32_t i = 0; i < n; ++i) Aq[i] -= aj * q[i] + bj * qp[i];
            bj = orc_norm2(n, Aq);
            if (bj < REAL_EPS * 1e6) break;
            be[nb++] = bj;
            memcpy(qp, q, sz);
            memcpy(q, Aq, sz);
            double s = 1.0 / bj;
            for (int32_t i = 0; i < n; ++i) q[i] *= s;
        }
        double tmin = al[0], tmax = al[0];
        for (int i = 0; i < na; ++i) {
            double r = 0.0;
            if (i > 0) r += fabs(be[i - 1]);
            if (i < na - 1) r += fabs(be[i]);
            tmin = dmin(tmin, al[i] - r);
            tmax = dmax(tmax, al[i] + r);
        }
        lam_max = dmax(tmax, REAL_EPS);
        lam_min = tmin;
        if (lam_min <= REAL_EPS) {
            double mpd = INFINITY;
            for (int32_t i = 0; i < n; ++i)
                for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
                    if (ci[k] == i && v[k] > REAL_EPS) { mpd = dmin(mpd, v[k]); break; }
            if (mpd == INFINITY) mpd = REAL_EPS;
            lam_min = mpd * 0.5;
        }
        lam_min = dmax(lam_min, REAL_EPS);
        cond = lam_max / lam_min;
        free(q); free(qp); free(Aq);
    }
    /* bandwidth, nnz variance (:394-416) */
    int32_t bw = 0;
    for (int32_t i = 0; i < n; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) { int32_t d = abs(i - ci[k]); if (d > bw) bw = d; }
    double avg = (n > 0) ? (double)nnz / n : 0.0;
    double var = 0.0;
    if (n > 0) {
        double mean = (double)nnz / n;
        for (int32_t i = 0; i < n; ++i) { double d = (rp[i + 1] - rp[i]) - mean; var += d * d; }
        var /= n;
    }
    int pos = 0;
    for (int32_t i = 0; i < n; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) { if (v[k] > 0.0) ++pos; break; }
    double dsf = (double)pos / (n > 1 ? n : 1);
    double max_asym = 0.0;
    for (int32_t i = 0; i < (n < 200 ? n : 200); ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            int32_t j = ci[k];
            if (j == i) continue;
            max_asym = dmax(max_asym, fabs(v[k] - get_entry(rp, ci, v, j, i)));
        }
    double ods = (fro > REAL_EPS) ? max_asym / fro : 0.0;
    double grad = 0.0;
    for (int32_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) s += fabs(v[k]);
        grad = dmax(grad, s);
    }
    int dc = 0;
    for (int32_t i = 0; i < n; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) if (ci[k] == i) { ++dc; break; }
    double dfrac = (nnz == 0) ? 0.0 : (double)dc / nnz;
    int64_t lo = 0, hi = 0;
    for (int32_t i = 0; i < n; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) { if (ci[k] < i) ++lo; if (ci[k] > i) ++hi; }
    double lur = (hi > 0) ? (double)lo / (double)hi : 1.0;
    int nzd = 0;
    for (int32_t i = 0; i < n; ++i) {
        int found = 0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) { if (fabs(v[k]) <= 1e-15) ++nzd; found = 1; break; }
        if (!found) ++nzd;
    }
    double strong = 0.0;
    for (int32_t i = 0; i < n; ++i) {
        double rm = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) if (ci[k] != i) rm = dmax(rm, fabs(v[k]));
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] != i && fabs(v[k]) >= 0.25 * rm) strong += 1.0;
    }
    double coarsen = 1.0 / (1.0 + ((n > 0) ? strong / n : 0.0));
    int depth = (int)log2((double)n / 50.0);
    if (depth < 1) depth = 1;
    const double af = 2e-10, am = 5e-9;
    double it_easy = dmin(sqrt(cond) * 0.5, 5000.0);
    double it_hard = dmin(log(cond + 1.0) * 5.0, 200.0);
    double ep_easy = it_easy * (af * 2.0 * nnz + am * 2.0 * n * 8);
    double ep_hard = it_hard * (af * 2.0 * nnz + am * 2.0 * n * 8);
    /* SPD sample check (:196-217) */
    int sym_ok = 1;
    {
        int32_t samp = n < 200 ? n : 200;
        int32_t stride = (samp > 0 && n / samp > 1) ? n / samp : 1;
        for (int32_t i = 0; i < n && sym_ok; i += stride)
            for (int32_t k = rp[i]; k < rp[i + 1] && sym_ok; ++k) {
                int32_t j = ci[k];
                if (j == i) continue;
                double aij = v[k], aji = get_entry(rp, ci, v, j, i);
                if (fabs(aij - aji) > 1e-6 * (1.0 + fabs(aij))) sym_ok = 0;
            }
    }
    int pd = 1;
    for (int32_t i = 0; i < n && pd; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) { if (v[k] <= 0.0) pd = 0; break; }
    int spd = sym_ok && pd;
    double f[24] = {(double)n, (double)nnz, density, diag_dom, ods, fro, cond, (double)spd,
                    (double)bw, avg, var, dsf, ods, lam_max, dmax(lam_min, REAL_EPS), grad,
                    dfrac, lur, (double)nzd, 1.0, coarsen, (double)depth, ep_easy, ep_hard};
    memcpy(feat, f, sizeof(f));
    /* select_initial_state (:225-233) */
    int32_t s;
    if (spd && cond < 1e6 && diag_dom >= 0.8) s = HAMLSS_STATE_EASY;
    else if (cond >= 1e6 || diag_dom < 0.3) s = HAMLSS_STATE_HARD;
    else s = HAMLSS_STATE_MODERATE;
    if (initial_state) *initial_state = s;
    return HAMLSS_OK;
}

/* AdaptiveSelector::solve (adaptive_selector.cpp:298-394): escalate only when an attempt
 * returns unconverged, warm-starting from the current x; stats keep the last attempt
 * with its setup time counted twice (:350-351). */
int orc_solve_adaptive(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                       const double* b, double* x, const hamlss_params* p, hamlss_stats* st,
                       hamlss_escalation* log, int32_t log_cap, int32_t* n_log,
                       int32_t* initial_state) {
    double feat[24];
    int32_t state;
    orc_extract_features(n, rp, ci, v, feat, &state);
    if (initial_state) *initial_state = state;
    *n_log = 0;
    int solved = 0;
    for (;;) {
        int kind = state == HAMLSS_STATE_EASY ? HAMLSS_PREC_JACOBI
                 : state == HAMLSS_STATE_MODERATE ? HAMLSS_PREC_ILU : HAMLSS_PREC_AMG;
        int solver = state == HAMLSS_STATE_EASY ? HAMLSS_SOLVER_CG : HAMLSS_SOLVER_FGMRES;
        double t0 = now_s();
        int status;
        orc_prec* M = orc_prec_setup(kind, n, rp, ci, v, p, &status);
        double setup = now_s() - t0;
        if (status != HAMLSS_OK) return status;
        hamlss_stats a;
        memset(&a, 0, sizeof(a));
        a.setup_time_s = setup;
        a.state_used = state;
        int r = solver == HAMLSS_SOLVER_CG ? orc_cg(n, rp, ci, v, M, b, x, p, &a)
                                           : orc_fgmres(n, rp, ci, v, M, b, x, p, &a);
        orc_prec_free(M);
        if (r < 0) return r;
        solved = r;
        a.state_used = state;
        *st = a;
        st->setup_time_s += a.setup_time_s;
        if (solved || state == HAMLSS_STATE_HARD) break;
        int32_t ns = state + 1;
        if (*n_log < log_cap) {
            hamlss_escalation* e = &log[*n_log];
            e->at_iteration = a.iterations;
            e->from_state = state;
            e->to_state = ns;
            e->residual_at_escalation = a.final_residual;
            e->reason = 0;
        }
        ++*n_log;
        state = ns;
    }
    st->state_used = state;
    return solved;
}
