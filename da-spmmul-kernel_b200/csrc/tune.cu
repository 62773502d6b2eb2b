// tune.cu -- autotuner: per problem fingerprint, the measured-best design-
// space point.
//
// The reference has no selector: the caller passes alg (spmvspmm.h:57-58)
// and the DA-SpMM paper's heuristic is not shipped.  Here the candidates of
// the design space (work split x reduction x coarsening x chunk x pipeline)
// are timed on the device for the caller's own matrix, and the fastest is
// cached under the matrix's fingerprint: layout, nv, storage, nr, nnz and the
// row-length quantiles (p50, p90, p99, max) -- the quantities the choice
// depends on.  DASPMM_ALG_AUTO looks the cache up by (layout, nv, nr, nnz)
// and falls back to a rule of thumb for shapes never tuned.
#include "internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace daspmm {

namespace {

struct Key {
    int layout, nv, nr, nnz;
    bool operator<(const Key &o) const
    {
        return std::tie(layout, nv, nr, nnz) < std::tie(o.layout, o.nv, o.nr, o.nnz);
    }
};

struct Entry {
    daspmm_fingerprint fp;
    daspmm_config cfg;
    float us;
};

std::mutex g_mu;
std::map<Key, Entry> g_cache;

// Row-length histogram over power-of-two buckets (bucket b holds lengths in
// [2^(b-1), 2^b), bucket 0 the empty rows) and the maximum.
__global__ void k_row_hist(const int *__restrict__ rowPtr, int nr, unsigned long long *hist,
                           int *maxlen)
{
    __shared__ unsigned long long h[33];
    if (threadIdx.x < 33) h[threadIdx.x] = 0;
    __syncthreads();
    int m = 0;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < nr;
         r += (long long)gridDim.x * blockDim.x) {
        const int len = __ldg(rowPtr + r + 1) - __ldg(rowPtr + r);
        const int b = len <= 0 ? 0 : 32 - __clz(len);
        atomicAdd(h + b, 1ull);
        m = max(m, len);
    }
    __syncthreads();
    if (threadIdx.x < 33 && h[threadIdx.x]) atomicAdd(hist + threadIdx.x, h[threadIdx.x]);
    atomicMax(maxlen, m);
}

daspmm_status fingerprint(int layout, int nr, int nnz, int nv, int dtype, const int *rowPtr,
                          cudaStream_t st, daspmm_fingerprint *out)
{
    daspmm_fingerprint fp{};
    fp.layout = layout; fp.nv = nv; fp.dtype = dtype; fp.nr = nr; fp.nnz = nnz;
    if (nr > 0 && rowPtr) {
        unsigned long long *d_hist = nullptr;
        int *d_max = nullptr;
        void *blk = nullptr;
        daspmm_status s = cached_workspace(33 * sizeof(unsigned long long) + 256, st, &blk);
        if (s != DASPMM_OK) return s;
        d_hist = (unsigned long long *)blk;
        d_max = (int *)((char *)blk + 33 * sizeof(unsigned long long));
        cudaMemsetAsync(blk, 0, 33 * sizeof(unsigned long long) + sizeof(int), st);
        const unsigned g = (unsigned)std::min(1184, std::max(1, (nr + 255) / 256));
        k_row_hist<<<g, 256, 0, st>>>(rowPtr, nr, d_hist, d_max);
        count_launches(1);
        unsigned long long h[33];
        int mx = 0;
        cudaError_t e = cudaMemcpyAsync(h, d_hist, sizeof(h), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&mx, d_max, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e);
        fp.max_row = mx;
        // quantile q: upper edge of the first bucket whose cumulative count reaches q*nr
        const double qs[3] = {0.5, 0.9, 0.99};
        int *dst[3] = {&fp.p50, &fp.p90, &fp.p99};
        for (int k = 0; k < 3; ++k) {
            unsigned long long acc = 0;
            for (int b = 0; b < 33; ++b) {
                acc += h[b];
                if ((double)acc >= qs[k] * nr) {
                    *dst[k] = b == 0 ? 0 : std::min(mx, (1 << b) - 1);
                    break;
                }
            }
        }
    }
    *out = fp;
    return DASPMM_OK;
}

// Candidate design points for one shape.
std::vector<daspmm_config> candidates(int layout, int nv, bool have_coo)
{
    std::vector<daspmm_config> v;
    auto add = [&](int alg, int pipe = 0, int chunk = 0, int S = 0, int cf = 0, int L = 0) {
        daspmm_config c{};
        c.alg = alg; c.pipe = pipe; c.chunk = chunk; c.lanes_nnz = S; c.cf = cf;
        c.lanes_col = L;
        v.push_back(c);
    };
    add(DASPMM_ALG_CSR_SCALAR);
    add(DASPMM_ALG_CSR_VECTOR);
    if (have_coo) {
        add(DASPMM_ALG_COO_SCALAR);
        add(DASPMM_ALG_COO_VECTOR);
    }
    if (layout == DASPMM_ROW_MAJOR && nv % 32 == 0) {
        // the window kernel: chunk sizes at the widest tile, then narrower
        // column tiles (64 / 32 floats: G = 8 / the 32-lane kernel)
        for (int ch : {64, 96, 128, 256}) add(DASPMM_ALG_CSR_BALANCED, 4, ch);
        for (int L : {16, 8})
            if (nv % (4 * L) == 0 && (nv % 128 == 0 || (L == 8 && nv % 64 == 0)))
                for (int ch : {64, 128}) add(DASPMM_ALG_CSR_BALANCED, 4, ch, 0, 0, L);
        add(DASPMM_ALG_CSR_BALANCED, 3);
        add(DASPMM_ALG_CSR_BALANCED, 2);
        add(DASPMM_ALG_CSR_BALANCED, 1);
    } else {
        for (int ch : {32, 128}) add(DASPMM_ALG_CSR_BALANCED, 1, ch);
        if (layout == DASPMM_ROW_MAJOR && nv <= 8) {
            add(DASPMM_ALG_CSR_VECTOR, 0, 0, 4);
            add(DASPMM_ALG_CSR_VECTOR, 0, 0, 8);
        }
        if (layout == DASPMM_COL_MAJOR)
            for (int cf : {2, 4, 8}) add(DASPMM_ALG_CSR_SCALAR, 0, 0, 0, cf);
    }
    if (layout == DASPMM_COL_MAJOR && nv >= 4) {  // through a row-major product
        add(DASPMM_ALG_CSR_BALANCED, 5);
        add(DASPMM_ALG_CSR_BALANCED, 5, 256);
    }
    return v;
}

float time_config(const daspmm_config &c, int layout, int nr, int nc, int nnz, int nv,
                  const int *rowPtr, const int *rowIdx, const int *colIdx, const float *values,
                  const float *B, float *C, int reps, cudaStream_t st, bool *ok)
{
    *ok = false;
    for (int i = 0; i < 2; ++i)
        if (daspmm_spmm_ex(&c, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values, B, C,
                           0.0f, nullptr, 0, st) != DASPMM_OK)
            return 0.0f;
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return 0.0f;
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return 0.0f;
    }
    cudaEventRecord(a, st);
    bool good = true;
    for (int i = 0; i < reps && good; ++i)
        good = daspmm_spmm_ex(&c, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values, B, C,
                              0.0f, nullptr, 0, st) == DASPMM_OK;
    cudaEventRecord(b, st);
    float ms = 0.0f;
    const bool done = cudaEventSynchronize(b) == cudaSuccess &&
                      cudaEventElapsedTime(&ms, a, b) == cudaSuccess;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ok = good && done;
    return ms * 1000.0f / reps;
}

}  // namespace

daspmm_status tuned_config(int layout, int nr, int nc, int nnz, int nv, daspmm_config *out)
{
    (void)nc;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_cache.find(Key{layout, nv, nr, nnz});
        if (it != g_cache.end()) {
            *out = it->second.cfg;
            return DASPMM_OK;
        }
    }
    // Rule of thumb for untuned shapes: the balanced split for wide dense
    // operands (B rows of >= 128 bytes), the row-balanced scalar kernel
    // otherwise.
    daspmm_config c{};
    c.alg = (layout == DASPMM_ROW_MAJOR && nv >= 32) ? DASPMM_ALG_CSR_BALANCED
                                                      : DASPMM_ALG_CSR_SCALAR;
    Resolved r;
    daspmm_status s = resolve(&c, layout, nr, nc, nnz, nv, nullptr, nullptr, &r);
    if (s != DASPMM_OK) return s;
    *out = to_config(r);
    return DASPMM_OK;
}

}  // namespace daspmm

using namespace daspmm;

extern "C" {

daspmm_status daspmm_fingerprint_of(int layout, int nr, int nnz, int nv, int dtype,
                                    const int *rowPtr, void *stream, daspmm_fingerprint *out)
{
    if (!out || nr < 0 || nnz < 0 || nv < 1) return DASPMM_ERR_INVALID;
    return fingerprint(layout, nr, nnz, nv, dtype, rowPtr, (cudaStream_t)stream, out);
}

daspmm_status daspmm_autotune(int layout, int nr, int nc, int nnz, int nv, const int *rowPtr,
                              const int *rowIdx, const int *colIdx, const float *values,
                              const float *B, float *C, int reps, daspmm_config *best,
                              float *best_us, void *stream)
{
    if (nr < 0 || nnz < 0 || nv < 1 || !rowPtr || !B || !C) return DASPMM_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    daspmm_fingerprint fp;
    daspmm_status s = fingerprint(layout, nr, nnz, nv, DASPMM_F32, rowPtr, st, &fp);
    if (s != DASPMM_OK) return s;
    if (reps < 1) reps = 5;
    float bus = 0.0f;
    daspmm_config bcfg{};
    bool found = false;
    for (const daspmm_config &c0 : candidates(layout, nv, rowIdx != nullptr)) {
        // resolve to the concrete point (so the cache holds explicit values)
        Resolved r;
        if (resolve(&c0, layout, nr, nc, nnz, nv, B, C, &r) != DASPMM_OK) continue;
        const daspmm_config c = to_config(r);
        bool ok = false;
        const float us = time_config(c, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values,
                                     B, C, reps, st, &ok);
        if (!ok) {
            cudaGetLastError();
            continue;
        }
        if (!found || us < bus) {
            bus = us;
            bcfg = c;
            found = true;
        }
    }
    if (!found) return DASPMM_ERR_UNSUPPORTED;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_cache[Key{layout, nv, nr, nnz}] = Entry{fp, bcfg, bus};
    }
    if (best) *best = bcfg;
    if (best_us) *best_us = bus;
    return DASPMM_OK;
}

daspmm_status daspmm_tune_save(const char *path)
{
    if (!path) return DASPMM_ERR_INVALID;
    FILE *f = std::fopen(path, "w");
    if (!f) return DASPMM_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g_mu);
    std::fprintf(f, "# daspmm autotune cache v1\n");
    for (const auto &kv : g_cache) {
        const Entry &e = kv.second;
        const daspmm_config &c = e.cfg;
        std::fprintf(f, "%d %d %d %d %d %d %d %d %d %.3f %d %d %d %d %d %d %d %d %d\n",
                     e.fp.layout, e.fp.nv, e.fp.dtype, e.fp.nr, e.fp.nnz, e.fp.p50, e.fp.p90,
                     e.fp.p99, e.fp.max_row, e.us, c.alg, c.vec, c.lanes_col, c.lanes_nnz, c.cf,
                     c.chunk, c.snap, c.block, c.pipe);
    }
    std::fclose(f);
    return DASPMM_OK;
}

daspmm_status daspmm_tune_load(const char *path)
{
    if (!path) return DASPMM_ERR_INVALID;
    FILE *f = std::fopen(path, "r");
    if (!f) return DASPMM_ERR_INVALID;
    char line[512];
    int n = 0;
    std::lock_guard<std::mutex> lk(g_mu);
    while (std::fgets(line, sizeof line, f)) {
        if (line[0] == '#') continue;
        Entry e{};
        daspmm_config &c = e.cfg;
        if (std::sscanf(line, "%d %d %d %d %d %d %d %d %d %f %d %d %d %d %d %d %d %d %d",
                        &e.fp.layout, &e.fp.nv, &e.fp.dtype, &e.fp.nr, &e.fp.nnz, &e.fp.p50,
                        &e.fp.p90, &e.fp.p99, &e.fp.max_row, &e.us, &c.alg, &c.vec, &c.lanes_col,
                        &c.lanes_nnz, &c.cf, &c.chunk, &c.snap, &c.block, &c.pipe) == 19) {
            g_cache[Key{e.fp.layout, e.fp.nv, e.fp.nr, e.fp.nnz}] = e;
            ++n;
        }
    }
    std::fclose(f);
    return n > 0 ? DASPMM_OK : DASPMM_ERR_INVALID;
}

void daspmm_tune_clear(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_cache.clear();
}

}  // extern "C"
