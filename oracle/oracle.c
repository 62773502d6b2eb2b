/*
 * oracle.c -- CPU restatement of the reference's host arithmetic for the
 * SpMM/SpMV path (see oracle.h).  TEST INFRASTRUCTURE ONLY: the checker, never
 * the thing measured or shipped.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fPIC -shared).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* generateCsrRowPtrArray (spmvspmm_benchmark.cu:41-76)                      */
/* ------------------------------------------------------------------------ */
int or_coo_to_csr_rowptr(int nr, int nnz, const int *rowIdx, int *rowPtr)
{
    /* The reference walks the sorted row list once, writing the current
     * position into every row pointer it passes (:63-73).  The same result
     * is: rowPtr[r] = number of nonzeros whose row is < r. */
    int p = 0;
    for (int r = 0; r <= nr; ++r) {
        while (p < nnz && rowIdx[p] < r) {
            if (p > 0 && rowIdx[p] < rowIdx[p - 1]) return -1;
            if (rowIdx[p] < 0) return -1;
            ++p;
        }
        rowPtr[r] = p;
    }
    if (p != nnz) return -1; /* a row index >= nr */
    return 0;
}

/* ------------------------------------------------------------------------ */
/* cpuSpmvReference (spmvspmm_benchmark.cu:11-39)                            */
/* ------------------------------------------------------------------------ */
void or_spmm_f32(int layout, int nr, int nc, int nnz, int nv,
                 const int *rowPtr, const int *colIdx, const float *values,
                 const float *B, float *C)
{
    (void)nnz;
    if (layout == OR_COL_MAJOR) {
        /* :15-24 -- dense column k outer, then rows, then the row's nonzeros */
        for (int k = 0; k < nv; ++k) {
            const float *vec = B + (size_t)k * nc;
            for (int r = 0; r < nr; ++r) {
                float val = 0.0f;
                for (int p = rowPtr[r]; p < rowPtr[r + 1]; ++p)
                    val += values[p] * vec[colIdx[p]];
                C[(size_t)k * nr + r] = val;
            }
        }
    } else {
        /* :27-37 -- per row a zeroed accumulator of nv floats; nonzeros outer,
         * dense columns inner. */
        float *vals = (float *)malloc(sizeof(float) * (size_t)(nv > 0 ? nv : 1));
        for (int r = 0; r < nr; ++r) {
            for (int k = 0; k < nv; ++k) vals[k] = 0.0f;
            for (int p = rowPtr[r]; p < rowPtr[r + 1]; ++p) {
                const float a = values[p];
                const float *brow = B + (size_t)colIdx[p] * nv;
                for (int k = 0; k < nv; ++k) vals[k] += a * brow[k];
            }
            for (int k = 0; k < nv; ++k) C[(size_t)r * nv + k] = vals[k];
        }
        free(vals);
    }
}

static void spmm_f64_core(int layout, int nr, int nc, int nv, const int *rowPtr,
                          const int *colIdx, const float *vf, const double *vd,
                          const float *Bf, const double *Bd, double *C,
                          double *absC)
{
    for (int r = 0; r < nr; ++r) {
        for (int k = 0; k < nv; ++k) {
            double s = 0.0, a = 0.0;
            for (int p = rowPtr[r]; p < rowPtr[r + 1]; ++p) {
                const int col = colIdx[p];
                const size_t bi = layout == OR_COL_MAJOR ? (size_t)k * nc + col
                                                         : (size_t)col * nv + k;
                const double x = vf ? (double)vf[p] : vd[p];
                const double y = Bf ? (double)Bf[bi] : Bd[bi];
                s += x * y;
                a += fabs(x) * fabs(y);
            }
            const size_t ci = layout == OR_COL_MAJOR ? (size_t)k * nr + r
                                                     : (size_t)r * nv + k;
            C[ci] = s;
            if (absC) absC[ci] = a;
        }
    }
}

void or_spmm_f64(int layout, int nr, int nc, int nnz, int nv,
                 const int *rowPtr, const int *colIdx, const float *values,
                 const float *B, double *C, double *absC)
{
    (void)nnz;
    spmm_f64_core(layout, nr, nc, nv, rowPtr, colIdx, values, NULL, B, NULL, C,
                  absC);
}

void or_spmm_f64d(int layout, int nr, int nc, int nnz, int nv,
                  const int *rowPtr, const int *colIdx, const double *values,
                  const double *B, double *C, double *absC)
{
    (void)nnz;
    spmm_f64_core(layout, nr, nc, nv, rowPtr, colIdx, NULL, values, NULL, B, C,
                  absC);
}

/* ------------------------------------------------------------------------ */
/* checkResult (spmvspmm_benchmark.cu:93-116)                                */
/* ------------------------------------------------------------------------ */
int or_check_result(int host_layout, int dev_layout, int nrows, int ncols,
                    const float *ref, const float *out, float eps,
                    int first_only, int *bad_i, int *bad_j)
{
    int passed = 1;
    for (int i = 0; i < nrows; ++i) {
        for (int j = 0; j < ncols; ++j) {
            const size_t i1 = host_layout == OR_ROW_MAJOR ? (size_t)i * ncols + j
                                                          : (size_t)j * nrows + i;
            const size_t i2 = dev_layout == OR_ROW_MAJOR ? (size_t)i * ncols + j
                                                         : (size_t)j * nrows + i;
            /* the reference fails on |out-ref| > eps (:103); a NaN also fails
             * here, where the reference's comparison would let it pass */
            const float d = fabsf(out[i2] - ref[i1]);
            if (!(d <= eps)) {
                if (passed) {
                    if (bad_i) *bad_i = i;
                    if (bad_j) *bad_j = j;
                }
                passed = 0;
                if (first_only) return 0;
                break; /* the reference moves on to the next row (:109) */
            }
        }
    }
    return passed;
}

/* ------------------------------------------------------------------------ */
/* calcMaxNv (spmvspmm_benchmark.cu:78-90)                                   */
/* ------------------------------------------------------------------------ */
int or_calc_max_nv(int nr, int nc, int nnz, size_t mem_bytes, int dtype_size,
                   int maxnv)
{
    const size_t sp = ((size_t)nr + 1 + (size_t)nnz + (size_t)nnz) * sizeof(int) +
                      (size_t)nnz * (size_t)dtype_size;
    const long long maxv = mem_bytes > sp
        ? (long long)((mem_bytes - sp) / (size_t)dtype_size / ((size_t)nr + nc))
        : 0;
    int nv = maxnv;
    while (nv > maxv && nv > 0) nv /= 2;
    return nv;
}

/* ------------------------------------------------------------------------ */
/* Partition arithmetic                                                      */
/* ------------------------------------------------------------------------ */
int or_row_of(const int *rowPtr, int nr, int k)
{
    /* first index in rowPtr[0..nr] with rowPtr[i] > k, minus one */
    int lo = 0, hi = nr + 1;
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (rowPtr[mid] <= k) lo = mid + 1;
        else hi = mid;
    }
    return lo - 1;
}

int or_num_chunks(int nnz, int chunk)
{
    if (chunk <= 0) return -1;
    const int n = (int)(((long long)nnz + chunk - 1) / chunk);
    return n > 0 ? n : 1;
}

void or_balanced_partition(int nr, int nnz, const int *rowPtr, int chunk,
                           int snap, int *meta)
{
    const int nch = or_num_chunks(nnz, chunk);
    meta[0] = 0;
    meta[1] = 0;
    for (int c = 1; c < nch; ++c) {
        const int k = (int)((long long)c * chunk);
        const int s = or_row_of(rowPtr, nr, k); /* row containing nonzero k */
        const int rs = rowPtr[s], re = rowPtr[s + 1];
        int kk = k;
        if (k > rs && re - rs < snap) kk = rs;
        meta[2 * c] = kk;
        meta[2 * c + 1] = s;
    }
    meta[2 * nch] = nnz;
    meta[2 * nch + 1] = nr;
}

int or_balanced_ownership(int nr, int nnz, const int *rowPtr, int chunk,
                          int snap, int *owner)
{
    const int nch = or_num_chunks(nnz, chunk);
    int *meta = (int *)malloc(sizeof(int) * 2 * (size_t)(nch + 1));
    or_balanced_partition(nr, nnz, rowPtr, chunk, snap, meta);
    for (int r = 0; r < nr; ++r) { owner[2 * r] = -1; owner[2 * r + 1] = 0; }
    int bad = 0;
    for (int c = 0; c < nch; ++c) {
        const int k0 = meta[2 * c], s0 = meta[2 * c + 1];
        const int k1 = meta[2 * c + 2], s1 = meta[2 * c + 3];
        int r = s0;
#define OR_FINISH(row)                                                      \
    do {                                                                    \
        if ((row) < 0 || (row) >= nr) { bad = 1; break; }                   \
        owner[2 * (row) + 1] += 1;                                          \
        if (rowPtr[(row)] >= k0) {                                          \
            if (owner[2 * (row)] != -1) bad = 1;                            \
            owner[2 * (row)] = c;                                           \
        }                                                                   \
    } while (0)
        for (int p = k0; p < k1; ++p) {
            while (p >= rowPtr[r + 1]) { OR_FINISH(r); ++r; }
        }
        while (r < s1) { OR_FINISH(r); ++r; }
        if (r < nr && r == s1 && rowPtr[r] < k1) OR_FINISH(r);
#undef OR_FINISH
    }
    for (int r = 0; r < nr; ++r)
        if (owner[2 * r] < 0 || owner[2 * r + 1] < 1) bad = 1;
    free(meta);
    return bad ? -1 : 0;
}

int or_coo_ownership(int nr, int nnz, const int *rowIdx, int chunk, int *owner)
{
    for (int r = 0; r < nr; ++r) { owner[2 * r] = -1; owner[2 * r + 1] = 0; }
    if (nnz == 0) return 0;
    const int nch = or_num_chunks(nnz, chunk);
    for (int c = 0; c < nch; ++c) {
        const long long k0 = (long long)c * chunk;
        const long long k1 = k0 + chunk < nnz ? k0 + chunk : nnz;
        int prev = -1;
        for (long long p = k0; p < k1; ++p) {
            const int r = rowIdx[p];
            if (r < 0 || r >= nr) return -1;
            if (r != prev) {
                owner[2 * r + 1] += 1;
                if (owner[2 * r] == -1) owner[2 * r] = c;
                prev = r;
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Reduced-precision formats                                                 */
/* ------------------------------------------------------------------------ */
static uint32_t f2u(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
static float u2f(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }

uint16_t or_f32_to_bf16(float x)
{
    uint32_t u = f2u(x);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);
    u += 0x7fffu + ((u >> 16) & 1u); /* round to nearest, ties to even */
    return (uint16_t)(u >> 16);
}

float or_bf16_to_f32(uint16_t h) { return u2f((uint32_t)h << 16); }

uint16_t or_f32_to_f16(float x)
{
    _Float16 h = (_Float16)x; /* IEEE conversion, round to nearest even */
    uint16_t u;
    memcpy(&u, &h, 2);
    return u;
}

float or_f16_to_f32(uint16_t u)
{
    _Float16 h;
    memcpy(&h, &u, 2);
    return (float)h;
}

float or_e4m3_to_f32(uint8_t v)
{
    const int s = v >> 7, e = (v >> 3) & 15, m = v & 7;
    if (e == 15 && m == 7) return NAN;
    const double mag = e == 0 ? ldexp((double)m, -9) : ldexp(1.0 + m / 8.0, e - 7);
    return (float)(s ? -mag : mag);
}

uint8_t or_f32_to_e4m3(float x)
{
    if (isnan(x)) return 0x7f;
    const uint8_t s = signbit(x) ? 0x80 : 0x00;
    const double a = fabs((double)x);
    if (a >= 448.0) return s | 0x7e; /* satfinite */
    if (a < ldexp(1.0, -6)) {
        /* subnormal range, spacing 2^-9; m == 8 encodes the smallest normal */
        const int m = (int)nearbyint(a * 512.0);
        return s | (uint8_t)m;
    }
    int E;
    const double f = frexp(a, &E); /* a = f * 2^E, f in [0.5, 1) */
    int e = E - 1;                 /* a = (2f) * 2^e, 2f in [1, 2) */
    int m = (int)nearbyint((2.0 * f - 1.0) * 8.0);
    if (m == 8) { m = 0; ++e; }
    const int be = e + 7;
    if (be > 15 || (be == 15 && m == 7)) return s | 0x7e;
    return s | (uint8_t)((be << 3) | m);
}

void or_quantize(int fmt, size_t n, const float *x, void *q)
{
    for (size_t i = 0; i < n; ++i) {
        switch (fmt) {
        case 0: ((float *)q)[i] = x[i]; break;
        case 1: ((uint16_t *)q)[i] = or_f32_to_bf16(x[i]); break;
        case 2: ((uint16_t *)q)[i] = or_f32_to_f16(x[i]); break;
        case 3: ((uint8_t *)q)[i] = or_f32_to_e4m3(x[i]); break;
        default: break;
        }
    }
}

void or_dequantize(int fmt, size_t n, const void *q, double *x)
{
    for (size_t i = 0; i < n; ++i) {
        switch (fmt) {
        case 0: x[i] = ((const float *)q)[i]; break;
        case 1: x[i] = or_bf16_to_f32(((const uint16_t *)q)[i]); break;
        case 2: x[i] = or_f16_to_f32(((const uint16_t *)q)[i]); break;
        case 3: x[i] = or_e4m3_to_f32(((const uint8_t *)q)[i]); break;
        default: x[i] = 0; break;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Seeded synthetic workloads.  The reference has no generator of its own (it */
/* reads SuiteSparse files, README.md:10, and fills B from a time(0)-seeded   */
/* rand(), helper.h:66-76).  These restate, step for step, the library's      */
/* generators (libdaspmm daspmm_gen_*) so that the benchmark's reference arm  */
/* builds the same inputs without loading the product library; a CPU test     */
/* checks them bit for bit against libdaspmm.                                 */
/* ------------------------------------------------------------------------ */
typedef struct { uint64_t s; } or_rng;

static uint64_t rng_next(or_rng *g)
{
    /* splitmix64 (Steele, Lea, Flood 2014) */
    uint64_t z = (g->s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static double rng_uniform(or_rng *g) { return (double)(rng_next(g) >> 11) * 0x1.0p-53; }
static float rng_unit24(or_rng *g) { return (float)(rng_next(g) >> 40) * 0x1.0p-24f; }
static uint32_t rng_below(or_rng *g, uint32_t n)
{
    return (uint32_t)(((rng_next(g) >> 32) * (uint64_t)n) >> 32);
}

#define OR_DEG_STREAM 0x243f6a8885a308d3ULL
#define OR_COL_STREAM 0x13198a2e03707344ULL
#define OR_VAL_STREAM 0xa4093822299f31d0ULL

static void gen_values(uint64_t seed, long long nnz, float *values)
{
    or_rng g = {seed ^ OR_VAL_STREAM};
    for (long long p = 0; p < nnz; ++p) values[p] = rng_unit24(&g) * 2.0f - 1.0f;
}

static int cmp_int(const void *a, const void *b)
{
    const int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* Column draw for one row: 0 = uniform over nc, 1 = preferential attachment
 * (an urn of every endpoint drawn so far, plus one entry per column). */
typedef struct { int kind, nc; const int *urn; size_t urn_n; } or_draw;

static int draw_col(or_rng *g, const or_draw *d)
{
    if (d->kind == 0) return (int)rng_below(g, (uint32_t)d->nc);
    const uint32_t u = rng_below(g, (uint32_t)(d->urn_n + (size_t)d->nc));
    return u < (uint32_t)d->nc ? (int)u : d->urn[u - (uint32_t)d->nc];
}

/* `deg` distinct columns for row r: up to 64 draws per column, then uniform
 * redraws; stamp[c] == r marks a column already taken; sorted ascending. */
static void distinct_row(int r, int deg, int nc, int *stamp, or_rng *g, const or_draw *d,
                         int *out)
{
    for (int j = 0; j < deg; ++j) {
        int col = -1;
        for (int tries = 0; tries < 64; ++tries) {
            const int c = draw_col(g, d);
            if (stamp[c] != r) { col = c; break; }
        }
        while (col < 0) {
            const int c = (int)rng_below(g, (uint32_t)nc);
            if (stamp[c] != r) col = c;
        }
        stamp[col] = r;
        out[j] = col;
    }
    qsort(out, (size_t)deg, sizeof(int), cmp_int);
}

int or_gen_uniform(int nr, int nc, int per_row, uint64_t seed, int *rowPtr, int *colIdx,
                   float *values)
{
    if (nr < 0 || nc < 1 || per_row < 0 || per_row > nc || !rowPtr) return -1;
    if ((long long)nr * per_row > 0x7fffffffLL) return -1;
    for (int r = 0; r <= nr; ++r) rowPtr[r] = r * per_row;
    if (!colIdx || !values) return 0;
    or_rng g = {seed ^ OR_COL_STREAM};
    int *stamp = (int *)malloc(sizeof(int) * (size_t)nc);
    if (!stamp) return -1;
    for (int c = 0; c < nc; ++c) stamp[c] = -1;
    const or_draw d = {0, nc, NULL, 0};
    for (int r = 0; r < nr; ++r)
        distinct_row(r, per_row, nc, stamp, &g, &d, colIdx + (size_t)r * per_row);
    free(stamp);
    gen_values(seed, (long long)nr * per_row, values);
    return 0;
}

int or_gen_powerlaw(int nr, int nc, double alpha, double shift, int dmin, int dmax,
                    double mean_scale, uint64_t seed, int *rowPtr, int *colIdx,
                    float *values, long long *nnz_out)
{
    if (nr < 0 || nc < 1 || dmin < 0 || dmax < dmin || !rowPtr || mean_scale <= 0) return -1;
    if (dmax > nc) dmax = nc;
    if (dmin > dmax) dmin = dmax;
    /* out-degree p(k) ~ (k + shift)^-alpha on [dmin, dmax], drawn by
     * inverting the normalised cumulative sum (first entry > u) */
    const int nk = dmax - dmin + 1;
    double *cdf = (double *)malloc(sizeof(double) * (size_t)nk);
    if (!cdf) return -1;
    double acc = 0;
    for (int k = dmin; k <= dmax; ++k) {
        acc += pow((double)k + shift, -alpha);
        cdf[k - dmin] = acc;
    }
    for (int i = 0; i < nk; ++i) cdf[i] /= acc;
    or_rng gd = {seed ^ OR_DEG_STREAM};
    long long nnz = 0;
    rowPtr[0] = 0;
    for (int r = 0; r < nr; ++r) {
        const double u = rng_uniform(&gd);
        int lo = 0, hi = nk; /* first i with cdf[i] > u */
        while (lo < hi) {
            const int mid = lo + (hi - lo) / 2;
            if (cdf[mid] > u) hi = mid; else lo = mid + 1;
        }
        int k = dmin + lo;
        if (k > dmax) k = dmax;
        if (mean_scale != 1.0) {
            k = (int)lround(k * mean_scale);
            if (k > dmax) k = dmax;
            if (k < dmin) k = dmin;
        }
        nnz += k;
        if (nnz > 0x7fffffffLL) { free(cdf); return -1; }
        rowPtr[r + 1] = (int)nnz;
    }
    free(cdf);
    if (nnz_out) *nnz_out = nnz;
    if (!colIdx || !values) return 0;
    or_rng gc = {seed ^ OR_COL_STREAM};
    int *urn = (int *)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    int *stamp = (int *)malloc(sizeof(int) * (size_t)nc);
    if (!urn || !stamp) { free(urn); free(stamp); return -1; }
    for (int c = 0; c < nc; ++c) stamp[c] = -1;
    size_t urn_n = 0;
    for (int r = 0; r < nr; ++r) {
        const int p0 = rowPtr[r], deg = rowPtr[r + 1] - p0;
        const or_draw d = {1, nc, urn, urn_n};
        distinct_row(r, deg, nc, stamp, &gc, &d, colIdx + p0);
        for (int j = 0; j < deg; ++j) urn[urn_n++] = colIdx[p0 + j];
    }
    free(urn);
    free(stamp);
    gen_values(seed, nnz, values);
    return 0;
}

void or_gen_dense(size_t n, uint64_t seed, float lo, float hi, float *out)
{
    or_rng g = {seed ^ OR_VAL_STREAM};
    for (size_t i = 0; i < n; ++i) out[i] = lo + (hi - lo) * rng_unit24(&g);
}
