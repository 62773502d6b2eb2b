// gen.cpp -- deterministic synthetic sparse/dense inputs (host code).
//
// The reference reads SuiteSparse Matrix Market files (README.md:10) and fills
// B from a time(0)-seeded rand() (helper.h:66-76), so its runs are not
// reproducible.  These generators give seeded stand-ins with the shapes and
// distributions of the benchmark configurations: a uniform matrix with exactly
// k distinct columns per row, a power-law graph with preferential attachment,
// and an Erdos-Renyi-like uniform matrix.  All use splitmix64, so the output
// is identical on every platform for a seed.
#include "daspmm.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next()
    {
        uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }  // [0, 1)
    float unit24() { return (float)(next() >> 40) * 0x1.0p-24f; }     // [0, 1), exact in fp32
    uint32_t below(uint32_t n) { return (uint32_t)(((next() >> 32) * (uint64_t)n) >> 32); }
};

// Distinct stream per purpose so that the first (degree-only) call and the
// second (fill) call of a generator see the same degrees.
constexpr uint64_t kDegStream = 0x243f6a8885a308d3ULL;
constexpr uint64_t kColStream = 0x13198a2e03707344ULL;
constexpr uint64_t kValStream = 0xa4093822299f31d0ULL;

void fill_values(uint64_t seed, long long nnz, float *values)
{
    Rng rv(seed ^ kValStream);
    for (long long p = 0; p < nnz; ++p) values[p] = rv.unit24() * 2.0f - 1.0f;
}

// Draw `deg` distinct columns for row r with draw(), recording them in
// stamp[] (stamp[col] == r marks a column already taken in this row).
template <class Draw>
void distinct_cols(int r, int deg, int nc, std::vector<int> &stamp, Rng &rng, Draw draw,
                   int *out)
{
    for (int j = 0; j < deg; ++j) {
        int col = -1;
        for (int tries = 0; tries < 64; ++tries) {
            const int c = draw();
            if (stamp[c] != r) { col = c; break; }
        }
        while (col < 0) {  // fall back to uniform redraws
            const int c = (int)rng.below((uint32_t)nc);
            if (stamp[c] != r) col = c;
        }
        stamp[col] = r;
        out[j] = col;
    }
    std::sort(out, out + deg);
}

}  // namespace

extern "C" {

daspmm_status daspmm_gen_uniform(int nr, int nc, int per_row, uint64_t seed, int *rowPtr,
                                 int *colIdx, float *values)
{
    if (nr < 0 || nc < 1 || per_row < 0 || per_row > nc || !rowPtr) return DASPMM_ERR_INVALID;
    if ((long long)nr * per_row > 0x7fffffffLL) return DASPMM_ERR_INVALID;
    for (int r = 0; r <= nr; ++r) rowPtr[r] = r * per_row;
    if (!colIdx || !values) return DASPMM_OK;
    Rng rc(seed ^ kColStream);
    std::vector<int> stamp(nc, -1);
    for (int r = 0; r < nr; ++r)
        distinct_cols(r, per_row, nc, stamp, rc, [&] { return (int)rc.below((uint32_t)nc); },
                      colIdx + (size_t)r * per_row);
    fill_values(seed, (long long)nr * per_row, values);
    return DASPMM_OK;
}

daspmm_status daspmm_gen_powerlaw(int nr, int nc, double alpha, double shift, int dmin,
                                  int dmax, double mean_scale, uint64_t seed, int *rowPtr,
                                  int *colIdx, float *values, long long *nnz_out)
{
    if (nr < 0 || nc < 1 || dmin < 0 || dmax < dmin || !rowPtr || mean_scale <= 0)
        return DASPMM_ERR_INVALID;
    dmax = std::min(dmax, nc);
    dmin = std::min(dmin, dmax);
    // discrete power law p(k) ~ (k + shift)^-alpha on [dmin, dmax], by inversion
    std::vector<double> cdf(dmax - dmin + 1);
    double acc = 0;
    for (int k = dmin; k <= dmax; ++k) {
        acc += std::pow((double)k + shift, -alpha);
        cdf[k - dmin] = acc;
    }
    for (double &x : cdf) x /= acc;
    Rng rd(seed ^ kDegStream);
    long long nnz = 0;
    rowPtr[0] = 0;
    for (int r = 0; r < nr; ++r) {
        const double u = rd.uniform();
        int k = dmin + (int)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        if (k > dmax) k = dmax;
        if (mean_scale != 1.0) {
            k = (int)std::lround(k * mean_scale);
            k = std::max(dmin, std::min(dmax, k));
        }
        nnz += k;
        if (nnz > 0x7fffffffLL) return DASPMM_ERR_INVALID;
        rowPtr[r + 1] = (int)nnz;
    }
    if (nnz_out) *nnz_out = nnz;
    if (!colIdx || !values) return DASPMM_OK;
    // preferential attachment: P(col) ~ in-degree(col) + 1.  The urn holds
    // one entry per edge endpoint so far; a draw below nc is the "+1" part.
    Rng rc(seed ^ kColStream);
    std::vector<int> urn;
    urn.reserve((size_t)nnz);
    std::vector<int> stamp(nc, -1);
    for (int r = 0; r < nr; ++r) {
        const int p0 = rowPtr[r], deg = rowPtr[r + 1] - p0;
        distinct_cols(r, deg, nc, stamp, rc,
                      [&] {
                          const uint32_t u = rc.below((uint32_t)(urn.size() + (size_t)nc));
                          return u < (uint32_t)nc ? (int)u : urn[u - nc];
                      },
                      colIdx + p0);
        for (int j = 0; j < deg; ++j) urn.push_back(colIdx[p0 + j]);
    }
    fill_values(seed, nnz, values);
    return DASPMM_OK;
}

daspmm_status daspmm_gen_random(int nr, int nc, double avg_deg, uint64_t seed, int *rowPtr,
                                int *colIdx, float *values, long long *nnz_out)
{
    if (nr < 0 || nc < 1 || avg_deg < 0 || !rowPtr) return DASPMM_ERR_INVALID;
    Rng rd(seed ^ kDegStream);
    long long nnz = 0;
    rowPtr[0] = 0;
    const double el = std::exp(-avg_deg);
    for (int r = 0; r < nr; ++r) {
        int k;
        if (avg_deg <= 30.0) {  // Poisson by multiplication of uniforms
            k = -1;
            double prod = 1.0;
            do { ++k; prod *= rd.uniform(); } while (prod > el);
        } else {  // normal approximation for large means
            const double u1 = std::max(rd.uniform(), 1e-300), u2 = rd.uniform();
            const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
            k = std::max(0, (int)std::lround(avg_deg + std::sqrt(avg_deg) * z));
        }
        k = std::min(k, nc);
        nnz += k;
        if (nnz > 0x7fffffffLL) return DASPMM_ERR_INVALID;
        rowPtr[r + 1] = (int)nnz;
    }
    if (nnz_out) *nnz_out = nnz;
    if (!colIdx || !values) return DASPMM_OK;
    Rng rc(seed ^ kColStream);
    std::vector<int> stamp(nc, -1);
    for (int r = 0; r < nr; ++r) {
        const int p0 = rowPtr[r];
        distinct_cols(r, rowPtr[r + 1] - p0, nc, stamp, rc,
                      [&] { return (int)rc.below((uint32_t)nc); }, colIdx + p0);
    }
    fill_values(seed, nnz, values);
    return DASPMM_OK;
}

void daspmm_gen_dense(size_t n, uint64_t seed, float lo, float hi, float *out)
{
    Rng rv(seed ^ kValStream);
    for (size_t i = 0; i < n; ++i) out[i] = lo + (hi - lo) * rv.unit24();
}

}  // extern "C"
