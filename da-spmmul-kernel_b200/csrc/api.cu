// api.cu -- the C ABI of libdaspmm.so (include/daspmm.h): argument checks,
// design-space resolution, workspace management and kernel launches.
//
// The reference's dispatcher cudaSpmm<256,32> (spmvspmm.h:53-199) picks one
// of twelve kernel templates from (alg, layout, nv) with hard-wired grids.
// Here (alg, layout, nv) resolve to a point (V, L, S, CF, chunk, snap) of one
// parametrised kernel family (kernels.cuh); the default point per shape is
// chosen for B200 (16-byte accesses, one group per row or per chunk, column
// tiles on gridDim.y), and daspmm_spmm_ex takes any legal point.
#include "daspmm.h"
#include "kernels.cuh"
#include "gather_tma.cuh"
#include "gather_lean.cuh"
#include "internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

namespace daspmm {

thread_local int g_last_cuda = 0;

int device_sms()
{
    static std::mutex mu;
    static std::map<int, int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 148;
    }
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(dev);
    if (it != cache.end()) return it->second;
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        n = 148;
    }
    cache[dev] = n;
    return n;
}

static std::atomic<long long> g_launches{0};
// Kernel timer: library-owned event pairs, one per timed call.
static std::mutex g_timer_mu;
static std::vector<cudaEvent_t> g_t_start, g_t_stop;
static int g_t_next = 0;
static thread_local int t_cur = -1;

void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void timer_before(cudaStream_t st)
{
    t_cur = -1;
    std::lock_guard<std::mutex> lk(g_timer_mu);
    if (g_t_next >= (int)g_t_start.size()) return;
    t_cur = g_t_next++;
    if (cudaEventRecord(g_t_start[t_cur], st) != cudaSuccess) {
        cudaGetLastError();
        t_cur = -1;
    }
}

void timer_after(cudaStream_t st)
{
    if (t_cur < 0) return;
    std::lock_guard<std::mutex> lk(g_timer_mu);
    if (t_cur < (int)g_t_stop.size() && cudaEventRecord(g_t_stop[t_cur], st) != cudaSuccess)
        cudaGetLastError();
    t_cur = -1;
}

daspmm_status cuda_fail(cudaError_t e)
{
    g_last_cuda = (int)e;
    return DASPMM_ERR_CUDA;
}

static int pow2ceil(int x)
{
    int p = 1;
    while (p < x && p < (1 << 30)) p <<= 1;
    return p;
}
static bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }
static bool aligned(const void *p, size_t a) { return ((uintptr_t)p % a) == 0; }

// ---------------------------------------------------------------- resolve
daspmm_status resolve(const daspmm_config *cfg, int layout, int nr, int nc, int nnz, int nv,
                      const void *B, const void *C, Resolved *out)
{
    if (!cfg || !out) return DASPMM_ERR_INVALID;
    if (layout != DASPMM_ROW_MAJOR && layout != DASPMM_COL_MAJOR) return DASPMM_ERR_INVALID;
    if (cfg->alg < DASPMM_ALG_CSR_SCALAR || cfg->alg > DASPMM_ALG_CSR_BALANCED)
        return DASPMM_ERR_INVALID;
    if (nv < 1 || nr < 0 || nnz < 0 || nc < 0) return DASPMM_ERR_INVALID;
    Resolved r{};
    r.alg = cfg->alg;
    r.cm = layout == DASPMM_COL_MAJOR;
    r.nr = nr;
    r.nc = nc;
    r.nnz = nnz;
    if (cfg->pipe < 0 || cfg->pipe > 5) return DASPMM_ERR_INVALID;
    if (cfg->l2_window < 0 || cfg->l2_window > 1000) return DASPMM_ERR_INVALID;
    r.l2_window = cfg->l2_window;
    if (cfg->pipe == 5 && !(r.cm && cfg->alg == DASPMM_ALG_CSR_BALANCED))
        return DASPMM_ERR_UNSUPPORTED;
    // Column-major balanced CSR with 4 or more columns: transpose B to
    // row-major, run the row-major product, transpose C back (pipe 5).  A
    // column-major gather reads one 4-byte value of a 32-byte sector per
    // (nonzero, column); the row-major one reads whole rows of B.
    if (r.cm && cfg->alg == DASPMM_ALG_CSR_BALANCED &&
        (cfg->pipe == 5 || (cfg->pipe == 0 && nv >= 4 && !cfg->vec && !cfg->cf &&
                            !cfg->lanes_col && !cfg->lanes_nnz))) {
        r.pipe = 5;
        r.inner_chunk = cfg->chunk;
        r.V = 1; r.L = 1; r.S = 1; r.CF = 1;
        r.chunk = cfg->chunk;
        r.nchunks = 0;
        r.snap = cfg->snap;
        r.block = 256;
        r.tiles = 1;
        *out = r;
        return DASPMM_OK;
    }
    const bool vector = cfg->alg == DASPMM_ALG_CSR_VECTOR || cfg->alg == DASPMM_ALG_COO_VECTOR;
    // vector width
    if (r.cm) {
        if (cfg->vec > 1) return DASPMM_ERR_UNSUPPORTED;
        r.V = 1;
    } else if (cfg->vec) {
        if (cfg->vec != 1 && cfg->vec != 2 && cfg->vec != 4) return DASPMM_ERR_INVALID;
        if (nv % cfg->vec) return DASPMM_ERR_INVALID;
        if (B && !aligned(B, 4 * cfg->vec)) return DASPMM_ERR_INVALID;
        if (C && !aligned(C, 4 * cfg->vec)) return DASPMM_ERR_INVALID;
        r.V = cfg->vec;
    } else {
        r.V = 1;
        if (nv % 4 == 0 && (!B || aligned(B, 16)) && (!C || aligned(C, 16))) r.V = 4;
        else if (nv % 2 == 0 && (!B || aligned(B, 8)) && (!C || aligned(C, 8))) r.V = 2;
    }
    const int vecs = (nv + r.V - 1) / r.V;  // vectors across a dense row
    // coarsening factor
    if (cfg->cf) r.CF = cfg->cf;
    else if (r.cm) r.CF = std::min(8, pow2ceil(nv));
    else r.CF = (!vector && vecs > 32) ? 2 : 1;
    if (r.cm ? !(r.CF == 1 || r.CF == 2 || r.CF == 4 || r.CF == 8)
             : !(r.CF == 1 || r.CF == 2))
        return DASPMM_ERR_UNSUPPORTED;
    // lanes across columns / nonzeros
    if (r.cm) {
        r.L = 1;
        if (cfg->lanes_col > 1) return DASPMM_ERR_UNSUPPORTED;
    } else if (cfg->lanes_col) {
        r.L = cfg->lanes_col;
    } else {
        const int need = pow2ceil((vecs + r.CF - 1) / r.CF);
        r.L = std::min(vector ? 8 : 32, need);
    }
    if (cfg->lanes_nnz) r.S = cfg->lanes_nnz;
    else if (!vector) r.S = 1;
    else r.S = r.cm ? 32 : 32 / r.L;
    if (!is_pow2(r.L) || !is_pow2(r.S) || r.L * r.S > 32) return DASPMM_ERR_INVALID;
    if ((cfg->alg == DASPMM_ALG_COO_SCALAR || cfg->alg == DASPMM_ALG_CSR_BALANCED) && r.S != 1)
        return DASPMM_ERR_UNSUPPORTED;
    const int G = r.L * r.S;
    // chunks
    if (cfg->alg >= DASPMM_ALG_COO_SCALAR) {
        if (cfg->chunk) r.chunk = cfg->chunk;
        else if (cfg->alg == DASPMM_ALG_COO_VECTOR) r.chunk = std::max(64, 8 * r.S);
        else if (r.cm) r.chunk = 32;
        else r.chunk = G >= 32 ? 128 : (G >= 16 ? 64 : 32);
        if (r.chunk < 1) return DASPMM_ERR_INVALID;
        if (cfg->alg == DASPMM_ALG_COO_VECTOR && r.chunk % r.S) return DASPMM_ERR_INVALID;
        r.nchunks = (int)std::max<long long>(1, ((long long)nnz + r.chunk - 1) / r.chunk);
        r.snap = cfg->snap ? cfg->snap : r.chunk / 2;
        if (r.snap < 1) r.snap = 1;
        if (r.snap > r.chunk) r.snap = r.chunk;  // keeps snapped boundaries ordered
    }
    r.block = cfg->block ? cfg->block : 256;
    if (r.block != 128 && r.block != 256) return DASPMM_ERR_INVALID;  // __launch_bounds__(256)
    r.pipe = 1;
    r.W = 0;
    if (cfg->alg == DASPMM_ALG_CSR_BALANCED && !r.cm && cfg->pipe != 1) {
        // TMA ring: one warp per chunk, W-float tiles (16-byte accesses, one
        // vector per lane group slot); the explicit fields, if given, must agree
        // tile width: the widest of 128/64/32 floats dividing nv, or 4*lanes_col
        int Wt = nv % 128 == 0 ? 128 : (nv % 64 == 0 ? 64 : 32);
        if (cfg->lanes_col == 8 || cfg->lanes_col == 16 || cfg->lanes_col == 32)
            Wt = 4 * cfg->lanes_col;
        const bool ok = nv % Wt == 0 && (!B || aligned(B, 16)) && (!C || aligned(C, 16)) &&
                        (!cfg->vec || cfg->vec == 4) && (!cfg->cf || cfg->cf == 1) &&
                        (!cfg->lanes_col || cfg->lanes_col == Wt / 4) &&
                        (!cfg->lanes_nnz || cfg->lanes_nnz == 1);
        if (cfg->pipe >= 2 && !ok) return DASPMM_ERR_UNSUPPORTED;
        if (ok) {
            r.pipe = cfg->pipe ? cfg->pipe : 4;
            r.W = Wt;
            r.V = 4; r.CF = 1; r.L = r.W / 4; r.S = 1;
            r.block = r.pipe == 4 ? 256 : 128;
            if (!cfg->chunk) {
                if (r.pipe == 4) {
                    // measured on the 262k power-law and 1M random matrices: one
                    // 128-column tile runs best at 96 nonzeros per chunk (FP32
                    // 93.3 -> 88.6 us on the power-law matrix), one 64-column
                    // tile at 64 (56.8 -> 53.8 us), wider products (several
                    // tiles in flight) at 128
                    r.chunk = nv == 128 ? 96 : (nv == 64 ? 64 : 128);
                } else {
                    // rings: one wave of chunks over the resident warps (12 per SM)
                    const long long slots = (long long)device_sms() * 12;
                    r.chunk = (int)std::max<long long>(64, ((long long)nnz + slots - 1) / slots);
                }
                r.nchunks = (int)std::max<long long>(1, ((long long)nnz + r.chunk - 1) / r.chunk);
                r.snap = cfg->snap ? std::min(cfg->snap, r.chunk) : r.chunk / 2;
            }
        }
    }
    const int W = r.L * r.V * r.CF;
    r.tiles = (nv + W - 1) / W;
    if (r.tiles > 65535) return DASPMM_ERR_UNSUPPORTED;
    *out = r;
    return DASPMM_OK;
}

// The row-major product inside pipe 5.
static daspmm_status resolve_inner(const Resolved &r, int nv, const void *B, const void *C,
                                   Resolved *in)
{
    daspmm_config c{};
    c.alg = DASPMM_ALG_CSR_BALANCED;
    c.chunk = r.inner_chunk;
    return resolve(&c, DASPMM_ROW_MAJOR, r.nr, r.nc, r.nnz, nv, B, C, in);
}

size_t workspace_bytes(const Resolved &r, int nv)
{
    if (r.pipe == 5) {  // [B row-major | C row-major | the row-major product's own]
        Resolved in;
        if (resolve_inner(r, nv, nullptr, nullptr, &in) != DASPMM_OK) return 0;
        return align256(sizeof(float) * (size_t)r.nc * nv) +
               align256(sizeof(float) * (size_t)r.nr * nv) + workspace_bytes(in, nv);
    }
    size_t b = 0;
    if (r.alg == DASPMM_ALG_CSR_BALANCED) {
        b += align256(sizeof(int2) * ((size_t)r.nchunks + 1));
        b += align256(sizeof(int) * (size_t)r.nchunks * r.tiles);  // split-row arrival counters
        b += align256(sizeof(unsigned int) * (size_t)r.tiles);     // chunk queue heads
        b += align256(sizeof(int) * ((size_t)r.nchunks + 1));      // chunks left to the walk
    }
    if (r.alg >= DASPMM_ALG_COO_SCALAR) b += align256(sizeof(float) * 2 * (size_t)r.nchunks * nv);
    return b;
}

// ---------------------------------------------------------------- launches
template <int W, int NS, int MODE>
static void launch_tma_w(const Resolved &r, const KArgs &a, cudaStream_t st)
{
    using R = TmaRing<W, NS>;
    static bool attr = false;  // per process: the attribute is per function
    if (!attr) {
        cudaFuncSetAttribute(k_bal_tma<W, NS, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             R::kCtaBytes);
        attr = true;
    }
    const unsigned gx = (unsigned)std::max<long long>(
        1, std::min<long long>(((long long)a.nchunks + R::kWarps - 1) / R::kWarps, 148LL * 64));
    k_bal_tma<W, NS, MODE><<<dim3(gx, r.tiles), R::kWarps * 32, R::kCtaBytes, st>>>(a);
}

template <int MODE>
static void launch_ring(const Resolved &r, const KArgs &a, cudaStream_t st)
{
    if (r.W == 128) launch_tma_w<128, 4, MODE>(r, a, st);
    else if (r.W == 64) launch_tma_w<64, 4, MODE>(r, a, st);
    else launch_tma_w<32, 4, MODE>(r, a, st);
}

template <int W>
static void launch_lean_w(const Resolved &r, const KArgs &a, cudaStream_t st)
{
    launch_lean<W, float, float, false>(r, a, st);
}

static void launch_tma(const Resolved &r, const KArgs &a, cudaStream_t st)
{
    if (r.pipe == 4) {
        if (r.W == 128) launch_lean_w<128>(r, a, st);
        else if (r.W == 64) launch_lean_w<64>(r, a, st);
        else launch_lean_w<32>(r, a, st);
    } else if (r.pipe == 3) {
        launch_ring<1>(r, a, st);
    } else {
        launch_ring<0>(r, a, st);
    }
}

template <bool CM, int V, int CF>
static void launch_all(const Resolved &r, KArgs &a, dim3 grid, dim3 fix_grid, int block,
                       cudaStream_t st)
{
    const bool fix = a.nchunks > 1;
    // the main kernel (pipe 4: the window or walk kernel after k_partition)
    // sits between the optional timer events
    timer_before(st);
    switch (r.alg) {
    case DASPMM_ALG_CSR_SCALAR:
    case DASPMM_ALG_CSR_VECTOR:
        k_rb<CM, V, CF><<<grid, block, 0, st>>>(a);
        break;
    case DASPMM_ALG_COO_SCALAR:
        k_eb_coo_sr<CM, V, CF, false><<<grid, block, 0, st>>>(a);
        break;
    case DASPMM_ALG_COO_VECTOR:
        k_eb_coo_pr<CM, V, CF><<<grid, block, 0, st>>>(a);
        break;
    case DASPMM_ALG_CSR_BALANCED:
        if (r.pipe >= 2) launch_tma(r, a, st);
        else k_bal<CM, V, CF, false><<<grid, block, 0, st>>>(a);
        break;
    }
    timer_after(st);
    count_launches(1);
    if (fix && r.alg >= DASPMM_ALG_COO_SCALAR && !(r.alg == DASPMM_ALG_CSR_BALANCED && r.pipe == 4)) {
        if (r.alg == DASPMM_ALG_CSR_BALANCED) k_fix_bal<CM, V, CF><<<fix_grid, block, 0, st>>>(a);
        else k_fix_coo<CM, V, CF><<<fix_grid, block, 0, st>>>(a);
        count_launches(1);
    }
}

static daspmm_status dispatch(const Resolved &r, KArgs &a, dim3 grid, dim3 fix_grid,
                              cudaStream_t st)
{
    const int blk = r.block;
#define DASPMM_CASE(CMV, v, cf)                                                  \
    if (r.cm == CMV && r.V == v && r.CF == cf) {                                \
        launch_all<CMV, v, cf>(r, a, grid, fix_grid, blk, st);                  \
        return DASPMM_OK;                                                       \
    }
    DASPMM_CASE(false, 1, 1) DASPMM_CASE(false, 1, 2)
    DASPMM_CASE(false, 2, 1) DASPMM_CASE(false, 2, 2)
    DASPMM_CASE(false, 4, 1) DASPMM_CASE(false, 4, 2)
    DASPMM_CASE(true, 1, 1) DASPMM_CASE(true, 1, 2)
    DASPMM_CASE(true, 1, 4) DASPMM_CASE(true, 1, 8)
#undef DASPMM_CASE
    return DASPMM_ERR_UNSUPPORTED;
}

// dst (Cn x R, row-major) = transpose of src (R x Cn, row-major) + beta * dst.
static void launch_transpose(const float *src, long long R, long long Cn, float *dst, float beta,
                             cudaStream_t st)
{
    const long long tiles = ((R + 31) / 32) * ((Cn + 31) / 32);
    const unsigned g = (unsigned)std::max<long long>(
        1, std::min<long long>(tiles, (long long)device_sms() * 16));
    k_transpose<<<g, dim3(32, 8), 0, st>>>(src, R, Cn, dst, beta);
    count_launches(1);
}

static unsigned grid_x(long long units, int G, int block)
{
    const long long gpb = (long long)(block / 32) * (32 / G);
    long long g = (units + gpb - 1) / gpb;
    const long long cap = 148LL * 64;  // grid-stride beyond ~64 CTAs per SM
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (unsigned)g;
}

daspmm_status run_resolved(const Resolved &r, int layout, int nr, int nc, int nnz, int nv,
                           const int *rowPtr, const int *rowIdx, const int *colIdx,
                           const float *values, const float *B, float *C, float beta,
                           void *ws, size_t ws_bytes, cudaStream_t st)
{
    if (nr == 0) return DASPMM_OK;
    const bool coo = r.alg == DASPMM_ALG_COO_SCALAR || r.alg == DASPMM_ALG_COO_VECTOR;
    if (!C || !B) return DASPMM_ERR_INVALID;
    if (nnz > 0 && (!colIdx || !values)) return DASPMM_ERR_INVALID;
    if (coo ? (nnz > 0 && !rowIdx) : !rowPtr) return DASPMM_ERR_INVALID;
    if (nc <= 0 && nnz > 0) return DASPMM_ERR_INVALID;
    const size_t need = workspace_bytes(r, nv);
    if (need > ws_bytes || (need && !ws)) return DASPMM_ERR_WORKSPACE;

    if (r.pipe == 5) {
        float *Brm = (float *)ws;
        float *Crm = (float *)((char *)ws + align256(sizeof(float) * (size_t)nc * nv));
        char *iws = (char *)Crm + align256(sizeof(float) * (size_t)nr * nv);
        Resolved in;
        daspmm_status s = resolve_inner(r, nv, Brm, Crm, &in);
        if (s != DASPMM_OK) return s;
        // B column-major = an nv x nc row-major array; its transpose is row-major B
        launch_transpose(B, nv, nc, Brm, 0.0f, st);
        s = run_resolved(in, DASPMM_ROW_MAJOR, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values,
                         Brm, Crm, 0.0f, iws, workspace_bytes(in, nv), st);
        if (s != DASPMM_OK) return s;
        launch_transpose(Crm, nr, nv, C, beta, st);  // C = transpose + beta * C
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
    }

    KArgs a{};
    a.nr = nr; a.nc = nc; a.nnz = nnz; a.nv = nv;
    a.ldb = layout == DASPMM_COL_MAJOR ? nc : nv;
    a.ldc = layout == DASPMM_COL_MAJOR ? nr : nv;
    a.rowPtr = rowPtr; a.rowIdx = rowIdx; a.colIdx = colIdx; a.vals = values;
    a.B = B; a.C = C; a.beta = beta;
    a.L = r.L; a.S = r.S; a.chunk = r.chunk; a.nchunks = r.nchunks;
    a.l2_window = r.l2_window;
    a.b_bytes = sizeof(float) * (size_t)nc * nv;
    const int G = r.L * r.S;

    if (coo) {
        if (beta != 1.0f) {
            const size_t n = (size_t)nr * nv;
            const unsigned g = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32);
            k_scale<<<std::max(1u, g), 256, 0, st>>>(C, n, beta);
            count_launches(1);
        }
        a.beta = 1.0f;
        if (nnz == 0) {
            cudaError_t e = cudaGetLastError();
            return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
        }
        a.slots = (float *)ws;
    } else if (r.alg == DASPMM_ALG_CSR_BALANCED) {
        carve_balanced(r, ws, &a);
        launch_partition(r, nr, nnz, rowPtr, a, st);
    }
    const long long units =
        (r.alg == DASPMM_ALG_CSR_SCALAR || r.alg == DASPMM_ALG_CSR_VECTOR) ? nr : r.nchunks;
    dim3 grid(grid_x(units, G, r.block), r.tiles);
    dim3 fix_grid(grid_x(r.nchunks, r.L, r.block), r.tiles);
    daspmm_status s = dispatch(r, a, grid, fix_grid, st);
    if (s != DASPMM_OK) return s;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

bool run_planned(const Resolved &r, int nr, int nc, int nnz, int nv, const int *rowPtr,
                 const int *colIdx, const float *values, const float *B, float *C, void *ws,
                 unsigned long long call, cudaStream_t st)
{
    if (r.alg != DASPMM_ALG_CSR_BALANCED || r.cm || r.pipe != 4 || nr <= 0) return false;
    // chunks per group of the window kernel: 32 / (W / 8) workers per warp
    const int nw = r.W == 128 ? 2 : 4;
    const unsigned long long ngroups = ((unsigned long long)r.nchunks + nw - 1) / nw;
    KArgs a{};
    a.nr = nr; a.nc = nc; a.nnz = nnz; a.nv = nv;
    a.ldb = nv; a.ldc = nv;
    a.rowPtr = rowPtr; a.colIdx = colIdx; a.vals = values;
    a.B = B; a.C = C; a.beta = 0.0f;
    a.L = r.L; a.S = r.S; a.chunk = r.chunk; a.nchunks = r.nchunks;
    a.l2_window = r.l2_window;
    a.b_bytes = sizeof(float) * (size_t)nc * nv;
    a.list_mode = 2;  // the plan's fixed list of chunks with an empty row
    a.head_base = (unsigned int)(call * ngroups);  // claims of the calls before, mod 2^32
    carve_balanced(r, ws, &a);
    timer_before(st);
    bool ok = false;
    if (r.W == 128 && (ok = launch_grp<128, float, float>(r, a, st)))
        launch_walk_list<128, float, float>(r, a, st);
    else if (r.W == 64 && (ok = launch_grp<64, float, float>(r, a, st)))
        launch_walk_list<64, float, float>(r, a, st);
    timer_after(st);
    if (ok) count_launches(1);
    return ok;
}

void workspace_tables(const Resolved &r, void *ws, const int2 **meta, int **list)
{
    KArgs a{};
    carve_balanced(r, ws, &a);
    *meta = a.meta;
    *list = a.list;
}

void carve_and_partition(const Resolved &r, int nr, int nnz, const int *rowPtr, void *ws,
                         cudaStream_t st)
{
    KArgs a{};
    carve_balanced(r, ws, &a);
    launch_partition(r, nr, nnz, rowPtr, a, st);
}

void carve_balanced(const Resolved &r, void *ws, KArgs *a)
{
    char *p = (char *)ws;
    a->meta = (const int2 *)p;
    p += align256(sizeof(int2) * ((size_t)r.nchunks + 1));
    a->cnt = (int *)p;
    p += align256(sizeof(int) * (size_t)r.nchunks * r.tiles);
    a->head = (unsigned int *)p;
    p += align256(sizeof(unsigned int) * (size_t)r.tiles);
    a->list = (int *)p;
    p += align256(sizeof(int) * ((size_t)r.nchunks + 1));
    a->slots = (float *)p;
}

void launch_partition(const Resolved &r, int nr, int nnz, const int *rowPtr, const KArgs &a,
                      cudaStream_t st)
{
    // one thread per row (a grid-stride form over 2 or 4 CTAs per SM measured
    // equal or slower)
    const unsigned pg = (unsigned)std::max(1, (nr + 255) / 256);
    // programmatic dependent launch: the CTAs are scheduled while the previous
    // kernel drains (measured 2.4 us per back-to-back SpMM on the power-law
    // matrix); k_partition waits for it before touching memory
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(pg);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_partition, nr, nnz, rowPtr, (int)r.chunk, (int)r.snap,
                       (int)r.nchunks, const_cast<int2 *>(a.meta), a.cnt, (int)r.tiles, a.head,
                       a.list);
    count_launches(1);
}

// ---------------------------------------------------------------- workspace
struct WsKey {
    int dev;
    void *stream;
    int tag;  // 0 = kernel workspace, 1 = host-entry staging block
    bool operator<(const WsKey &o) const
    {
        if (dev != o.dev) return dev < o.dev;
        if (stream != o.stream) return stream < o.stream;
        return tag < o.tag;
    }
};
static std::mutex g_ws_mu;
static std::map<WsKey, std::pair<void *, size_t>> g_ws;

static daspmm_status cached_block(size_t need, cudaStream_t st, int tag, void **out)
{
    *out = nullptr;
    if (need == 0) return DASPMM_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e);
    std::lock_guard<std::mutex> lk(g_ws_mu);
    auto &slot = g_ws[WsKey{dev, (void *)st, tag}];
    if (slot.second < need) {
        if (slot.first) {
            e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return cuda_fail(e);
            cudaFree(slot.first);
            slot = {nullptr, 0};
        }
        void *p = nullptr;
        const size_t bytes = std::max(need, (size_t)1 << 20);
        e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            g_last_cuda = (int)e;
            return DASPMM_ERR_NOMEM;
        }
        slot = {p, bytes};
    }
    *out = slot.first;
    return DASPMM_OK;
}

daspmm_status cached_workspace(size_t need, cudaStream_t st, void **out)
{
    return cached_block(need, st, 0, out);
}

daspmm_status cached_host_staging(size_t need, cudaStream_t st, void **out)
{
    return cached_block(need, st, 1, out);
}

}  // namespace daspmm

using namespace daspmm;

// ======================================================================
// extern "C"
// ======================================================================
extern "C" {

daspmm_status daspmm_default_config(int alg, int layout, int nr, int nc, int nnz, int nv,
                                    daspmm_config *out)
{
    (void)nc;
    if (!out) return DASPMM_ERR_INVALID;
    if (alg == DASPMM_ALG_AUTO) return tuned_config(layout, nr, nc, nnz, nv, out);
    daspmm_config c{};
    c.alg = alg;
    Resolved r;
    daspmm_status s = resolve(&c, layout, nr, nc, nnz, nv, nullptr, nullptr, &r);
    if (s != DASPMM_OK) return s;
    *out = to_config(r);
    return DASPMM_OK;
}

size_t daspmm_workspace_bytes(const daspmm_config *cfg, int layout, int nr, int nc, int nnz,
                              int nv)
{
    Resolved r;
    if (resolve(cfg, layout, nr, nc, nnz, nv, nullptr, nullptr, &r) != DASPMM_OK) return 0;
    return workspace_bytes(r, nv);
}

daspmm_status daspmm_spmm_ex(const daspmm_config *cfg, int layout, int nr, int nc, int nnz,
                             int nv, const int *rowPtr, const int *rowIdx,
                             const int *colIdx, const float *values, const float *B,
                             float *C, float beta, void *workspace, size_t ws_bytes,
                             void *stream)
{
    Resolved r;
    daspmm_status s = resolve(cfg, layout, nr, nc, nnz, nv, B, C, &r);
    if (s != DASPMM_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    if (!workspace) {
        const size_t need = workspace_bytes(r, nv);
        s = cached_workspace(need, st, &workspace);
        if (s != DASPMM_OK) return s;
        ws_bytes = need;
    }
    return run_resolved(r, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values, B, C,
                        beta, workspace, ws_bytes, st);
}

daspmm_status daspmm_spmm(int alg, int layout, int nr, int nc, int nnz, int nv,
                          const int *rowPtr, const int *rowIdx, const int *colIdx,
                          const float *values, const float *B, float *C, float beta,
                          void *stream)
{
    daspmm_config c{};
    if (alg == DASPMM_ALG_AUTO) {
        daspmm_status s = tuned_config(layout, nr, nc, nnz, nv, &c);
        if (s != DASPMM_OK) return s;
    } else {
        c.alg = alg;
    }
    return daspmm_spmm_ex(&c, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values, B, C,
                          beta, nullptr, 0, stream);
}

int daspmm_compat_spmm(int alg, int layout, int nr, int nc, int nnz, int nv,
                       const int *rowPtr, const int *rowIdx, const int *colIdx,
                       const float *values, const float *dnInput, float *dnOutput)
{
    if (alg < DASPMM_ALG_CSR_SCALAR || alg > DASPMM_ALG_COO_VECTOR)
        return (int)cudaErrorInvalidValue;
    const float beta = (alg == DASPMM_ALG_COO_SCALAR || alg == DASPMM_ALG_COO_VECTOR) ? 1.0f : 0.0f;
    daspmm_status s = daspmm_spmm(alg, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values,
                                  dnInput, dnOutput, beta, nullptr);
    switch (s) {
    case DASPMM_OK: return (int)cudaSuccess;
    case DASPMM_ERR_CUDA: return g_last_cuda;
    case DASPMM_ERR_NOMEM: return (int)cudaErrorMemoryAllocation;
    default: return (int)cudaErrorInvalidValue;
    }
}

int daspmm_num_chunks(int nnz, int chunk)
{
    if (chunk <= 0 || nnz < 0) return -1;
    return (int)std::max<long long>(1, ((long long)nnz + chunk - 1) / chunk);
}

daspmm_status daspmm_partition(int nr, int nnz, const int *rowPtr, int chunk, int snap,
                               int *meta, void *stream)
{
    if (nr < 0 || nnz < 0 || chunk < 1 || snap < 1 || !rowPtr || !meta) return DASPMM_ERR_INVALID;
    const int nch = daspmm_num_chunks(nnz, chunk);
    const unsigned pg = (unsigned)std::max(1, (nr + 255) / 256);
    k_partition<<<pg, 256, 0, (cudaStream_t)stream>>>(nr, nnz, rowPtr, chunk, std::min(snap, chunk),
                                                      nch, (int2 *)meta, nullptr, 1, nullptr,
                                                      nullptr);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

daspmm_status daspmm_ownership(int alg, int nr, int nnz, const int *rowPtr, const int *rowIdx,
                               int chunk, int snap, int *owner, void *stream)
{
    if (nr < 0 || nnz < 0 || chunk < 1 || !owner) return DASPMM_ERR_INVALID;
    if (alg != DASPMM_ALG_CSR_BALANCED && alg != DASPMM_ALG_COO_SCALAR) return DASPMM_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    if (nr == 0) return DASPMM_OK;
    // owner[2r] = INT_MAX, owner[2r+1] = 0, then the recording walk
    k_own_init<<<(unsigned)std::max(1, (nr + 255) / 256), 256, 0, st>>>(owner, nr);
    KArgs a{};
    a.nr = nr; a.nnz = nnz; a.nv = 1; a.ldb = 1; a.ldc = 1;
    a.rowPtr = rowPtr; a.rowIdx = rowIdx;
    a.L = 32; a.S = 1; a.chunk = chunk;
    a.nchunks = daspmm_num_chunks(nnz, chunk);
    a.own = owner;
    void *meta = nullptr;
    if (alg == DASPMM_ALG_CSR_BALANCED) {
        if (!rowPtr) return DASPMM_ERR_INVALID;
        daspmm_status s = cached_workspace(sizeof(int2) * ((size_t)a.nchunks + 1), st, &meta);
        if (s != DASPMM_OK) return s;
        s = daspmm_partition(nr, nnz, rowPtr, chunk, snap, (int *)meta, stream);
        if (s != DASPMM_OK) return s;
        a.meta = (const int2 *)meta;
        k_bal<false, 1, 1, true><<<grid_x(a.nchunks, 32, 256), 256, 0, st>>>(a);
    } else {
        if (nnz > 0) {
            if (!rowIdx) return DASPMM_ERR_INVALID;
            k_eb_coo_sr<false, 1, 1, true><<<grid_x(a.nchunks, 32, 256), 256, 0, st>>>(a);
        }
    }
    k_own_fini<<<(unsigned)std::max(1, (nr + 255) / 256), 256, 0, st>>>(owner, nr);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

daspmm_status daspmm_coo_to_csr(int nr, int nnz, const int *rowIdx, int *rowPtr, void *stream)
{
    if (nr < 0 || nnz < 0 || !rowPtr || (nnz > 0 && !rowIdx)) return DASPMM_ERR_INVALID;
    const long long n = (long long)nnz + 1;
    const unsigned g = (unsigned)std::max<long long>(1, (n + 255) / 256);
    k_coo_to_csr<<<g, 256, 0, (cudaStream_t)stream>>>(nr, nnz, rowIdx, rowPtr);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

long long daspmm_launch_count(void) { return g_launches.load(); }

// The bounded mbarrier wait of the ring kernels, run on its own: one thread
// arms a barrier and waits on it with mbar_wait.  With `expire`, the barrier
// expects 16 transaction bytes that no copy will ever deliver (nothing is
// issued, so nothing is in flight), so the wait runs out after `polls` polls
// and sets the device error word; otherwise the thread's own arrival
// completes the phase.  out[0] = 1 if the wait returned success, else 0.
static __global__ void k_wait_probe(int polls, int expire, int *out)
{
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x != 0) return;
    const uint32_t b = smem_addr(&bar);
    mbar_init(b, 1);
    mbar_init_fence();
    if (expire) mbar_arrive_expect_tx(b, 16);
    else mbar_arrive(b);
    const bool ok = mbar_wait(b, 0, polls);
    mbar_inval(b);
    out[0] = ok ? 1 : 0;
}

daspmm_status daspmm_wait_probe(int polls, int expire, int *out, void *stream)
{
    if (polls < 1 || !out) return DASPMM_ERR_INVALID;
    k_wait_probe<<<1, 32, 0, (cudaStream_t)stream>>>(polls, expire ? 1 : 0, out);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

daspmm_status daspmm_l2_set_aside(size_t bytes)
{
    int dev = 0, maxp = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, dev);
    if (e != cudaSuccess) return cuda_fail(e);
    if (bytes > (size_t)maxp) bytes = (size_t)maxp;  // the device's largest set-aside
    e = cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, bytes);
    if (e == cudaSuccess && bytes == 0) e = cudaCtxResetPersistingL2Cache();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

daspmm_status daspmm_device_error(void)
{
    int v = 0, zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int));
    if (e == cudaSuccess && v) e = cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e);
    return v ? DASPMM_ERR_TIMEOUT : DASPMM_OK;
}

static void timer_release()
{
    for (cudaEvent_t e : g_t_start) cudaEventDestroy(e);
    for (cudaEvent_t e : g_t_stop) cudaEventDestroy(e);
    g_t_start.clear();
    g_t_stop.clear();
    g_t_next = 0;
}

daspmm_status daspmm_kernel_timer_begin(int n)
{
    if (n < 0) return DASPMM_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g_timer_mu);
    timer_release();
    for (int i = 0; i < n; ++i) {
        cudaEvent_t a, b;
        cudaError_t e = cudaEventCreate(&a);
        if (e == cudaSuccess) {
            e = cudaEventCreate(&b);
            if (e != cudaSuccess) cudaEventDestroy(a);
        }
        if (e != cudaSuccess) {
            timer_release();
            return cuda_fail(e);
        }
        g_t_start.push_back(a);
        g_t_stop.push_back(b);
    }
    return DASPMM_OK;
}

int daspmm_kernel_timer_end(float *ms_out, int n)
{
    std::lock_guard<std::mutex> lk(g_timer_mu);
    const int used = g_t_next;
    int ok = 0;
    for (int i = 0; i < used; ++i) {
        float ms = 0.0f;
        cudaError_t e = cudaEventSynchronize(g_t_stop[i]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, g_t_start[i], g_t_stop[i]);
        if (e != cudaSuccess) {
            g_last_cuda = (int)e;
            timer_release();
            return -1;
        }
        if (ms_out && i < n) ms_out[i] = ms;
        ++ok;
    }
    timer_release();
    return ok;
}

static daspmm_status spmm_host_impl(const daspmm_config *cfg, int layout, int nr, int nc,
                                    int nnz, int nv, const int *rowPtr, const int *rowIdx,
                                    const int *colIdx, const float *values, const float *B,
                                    float *C, float beta, void *stream, bool sync)
{
    Resolved r;
    daspmm_status s = resolve(cfg, layout, nr, nc, nnz, nv, nullptr, nullptr, &r);
    if (s != DASPMM_OK) return s;
    if (nr == 0) return DASPMM_OK;
    if (nr < 0 || nc < 0 || nnz < 0 || !B || !C) return DASPMM_ERR_INVALID;
    const bool coo = r.alg == DASPMM_ALG_COO_SCALAR || r.alg == DASPMM_ALG_COO_VECTOR;
    if (coo ? (nnz > 0 && !rowIdx) : !rowPtr) return DASPMM_ERR_INVALID;
    if (nnz > 0 && (!colIdx || !values)) return DASPMM_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    // one device block: [rowPtr | rowIdx | colIdx | values | B | C | workspace]
    const size_t b_rp = coo ? 0 : align256(sizeof(int) * ((size_t)nr + 1));
    const size_t b_ri = coo ? align256(sizeof(int) * (size_t)nnz) : 0;
    const size_t b_ci = align256(sizeof(int) * (size_t)nnz);
    const size_t b_va = align256(sizeof(float) * (size_t)nnz);
    const size_t b_B = align256(sizeof(float) * (size_t)nc * nv);
    const size_t b_C = align256(sizeof(float) * (size_t)nr * nv);
    const size_t b_ws = workspace_bytes(r, nv);
    const size_t total = b_rp + b_ri + b_ci + b_va + b_B + b_C + b_ws;
    void *blk = nullptr;
    s = cached_host_staging(total, st, &blk);
    if (s != DASPMM_OK) return s;
    char *p = (char *)blk;
    int *d_rp = coo ? nullptr : (int *)p; p += b_rp;
    int *d_ri = coo ? (int *)p : nullptr; p += b_ri;
    int *d_ci = (int *)p; p += b_ci;
    float *d_va = (float *)p; p += b_va;
    float *d_B = (float *)p; p += b_B;
    float *d_C = (float *)p; p += b_C;
    void *d_ws = b_ws ? (void *)p : nullptr;
    cudaError_t e = cudaSuccess;
#define DASPMM_H2D(dst, src, bytes)                                                  \
    if ((bytes) && e == cudaSuccess)                                                 \
        e = cudaMemcpyAsync((dst), (src), (bytes), cudaMemcpyHostToDevice, st);
    DASPMM_H2D(d_rp, rowPtr, coo ? 0 : sizeof(int) * ((size_t)nr + 1))
    DASPMM_H2D(d_ri, rowIdx, coo ? sizeof(int) * (size_t)nnz : 0)
    DASPMM_H2D(d_ci, colIdx, sizeof(int) * (size_t)nnz)
    DASPMM_H2D(d_va, values, sizeof(float) * (size_t)nnz)
    DASPMM_H2D(d_B, B, sizeof(float) * (size_t)nc * nv)
    DASPMM_H2D(d_C, C, beta != 0.0f ? sizeof(float) * (size_t)nr * nv : 0)
#undef DASPMM_H2D
    if (e != cudaSuccess) return cuda_fail(e);
    s = run_resolved(r, layout, nr, nc, nnz, nv, d_rp, d_ri, d_ci, d_va, d_B, d_C, beta, d_ws,
                     b_ws, st);
    if (s != DASPMM_OK) return s;
    e = cudaMemcpyAsync(C, d_C, sizeof(float) * (size_t)nr * nv, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && sync) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

daspmm_status daspmm_spmm_host(const daspmm_config *cfg, int layout, int nr, int nc, int nnz,
                               int nv, const int *rowPtr, const int *rowIdx, const int *colIdx,
                               const float *values, const float *B, float *C, float beta,
                               void *stream)
{
    return spmm_host_impl(cfg, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values, B, C,
                          beta, stream, true);
}

daspmm_status daspmm_spmm_host_async(const daspmm_config *cfg, int layout, int nr, int nc,
                                     int nnz, int nv, const int *rowPtr, const int *rowIdx,
                                     const int *colIdx, const float *values, const float *B,
                                     float *C, float beta, void *stream)
{
    return spmm_host_impl(cfg, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values, B, C,
                          beta, stream, false);
}

const char *daspmm_status_string(daspmm_status s)
{
    switch (s) {
    case DASPMM_OK: return "ok";
    case DASPMM_ERR_INVALID: return "invalid argument";
    case DASPMM_ERR_UNSUPPORTED: return "unsupported configuration";
    case DASPMM_ERR_CUDA: return "CUDA error";
    case DASPMM_ERR_NOMEM: return "device allocation failed";
    case DASPMM_ERR_WORKSPACE: return "workspace too small";
    case DASPMM_ERR_TIMEOUT: return "bounded wait expired";
    case DASPMM_ERR_BUDGET: return "request exceeds memory budget";
    case DASPMM_ERR_CANCELLED: return "request cancelled";
    case DASPMM_ERR_BAD_MATRIX: return "malformed sparse matrix";
    }
    return "unknown status";
}

int daspmm_last_cuda_error(void) { return g_last_cuda; }
int daspmm_abi_version(void) { return DASPMM_ABI_VERSION; }

}  // extern "C"
