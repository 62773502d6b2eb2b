// batch.cu -- many SpMMs of uneven sizes in one persistent launch.
//
// The reference runs one problem per cudaSpmm call (spmvspmm.h:53-199); a
// batch here is a table of instances (each its own CSR A, dense B and C, all
// with the same column count nv and storage formats).  A plan kernel cuts
// every instance into work items -- (instance, row tile, column tile) --
// where row tiles hold about `chunk` nonzeros and never split a row.  The
// persistent kernel's warps take items from a device queue (one atomic per
// item) and gather each item's rows like the lean balanced kernel: windows
// of 32 nonzeros, four B rows in flight, row ends from a lane cache.  Every
// output row is summed by one warp in nonzero order, so a result does not
// depend on what else is in the batch or on scheduling.
//
// daspmm_batch_run is one memset (the queue head) and one launch, so it can
// be captured into a CUDA graph (daspmm_batch_capture / _replay).
#include "gather_lean.cuh"
#include "internal.h"
#include "kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

namespace daspmm {

struct BatchInst {
    int nr, nc, nnz, nv;
    int ldb, ldc;
    int row_tiles;  // T = max(1, ceil(nnz / chunk))
    int col_tiles;  // ceil(nv / W)
    const int *rowPtr;
    const int *colIdx;
    const void *vals;
    const void *B;
    const float *bscale;
    float *C;
    float beta;
};

struct BatchItem {
    int inst, row0, row1, ctile;
};

// item g -> (instance, row tile t, column tile); row tile t starts at the row
// holding nonzero t*chunk (row 0 for t = 0) and ends where tile t+1 starts
// (nr for the last), so tiles cover every row exactly once.
static __global__ void k_batch_plan(const BatchInst *__restrict__ inst,
                                    const long long *__restrict__ item_begin, int ninst,
                                    int chunk, BatchItem *items, long long nitems)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nitems) return;
    int lo = 0, hi = ninst;  // last i with item_begin[i] <= g
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (item_begin[mid] <= g) lo = mid;
        else hi = mid;
    }
    const BatchInst I = inst[lo];
    const long long local = g - item_begin[lo];
    const int t = (int)(local / I.col_tiles), ct = (int)(local % I.col_tiles);
    auto row_start = [&](int tt) -> int {
        if (tt == 0) return 0;
        if (tt >= I.row_tiles) return I.nr;
        const int k = tt * chunk;  // < nnz: the row containing nonzero k
        int a = 0, b = I.nr;       // last r with rowPtr[r] <= k
        while (b - a > 1) {
            const int m = (a + b) / 2;
            if (__ldg(I.rowPtr + m) <= k) a = m;
            else b = m;
        }
        return a;
    };
    BatchItem it;
    it.inst = lo;
    it.row0 = row_start(t);
    it.row1 = row_start(t + 1);
    it.ctile = ct;
    items[g] = it;
}

// Rows [row0, row1) of one instance, column tile [tb0, tb0 + W): the lean
// windowed gather over whole rows (no carries).  Lanes whose columns lie at or
// past nv (nv % W != 0) load a clamped, in-bounds vector and store nothing.
template <int W, int U, typename TV, typename TB>
__device__ __forceinline__ void batch_rows(const BatchInst &I, int row0, int row1, int tb0,
                                           uint64_t pol_once)
{
    constexpr int VL = W / 32;
    constexpr bool SCALED = std::is_same<TB, fp8>::value;
    const int lane = threadIdx.x & 31;
    const int col = tb0 + lane * VL;
    const bool active = col < I.nv;
    const int colc = active ? col : I.nv - VL;  // nv % VL == 0 (checked on the host)
    const TB *Bl = reinterpret_cast<const TB *>(I.B) + colc;
    const TV *Av = reinterpret_cast<const TV *>(I.vals);
    float sc[VL];
#pragma unroll
    for (int e = 0; e < VL; ++e) sc[e] = SCALED ? __ldg(I.bscale + colc + e) : 1.0f;
    const int k0 = __ldg(I.rowPtr + row0), k1 = __ldg(I.rowPtr + row1);
    int r = row0, rb = r;
    int rc = __ldg(I.rowPtr + min(rb + 1 + lane, I.nr));
    int rn = __ldg(I.rowPtr + min(rb + 33 + lane, I.nr));
    int re = __shfl_sync(kFull, rc, 0);
    float acc[VL];
#pragma unroll
    for (int e = 0; e < VL; ++e) acc[e] = 0.0f;
    auto emit = [&](int row) {
        if (active) {
            float *dst = I.C + (size_t)row * I.ldc + col;
#pragma unroll
            for (int e = 0; e < VL; ++e) acc[e] *= sc[e];
            if (I.beta != 0.0f) {
                float old[VL];
                ld_plain<VL>(old, dst);
#pragma unroll
                for (int e = 0; e < VL; ++e) acc[e] = fmaf(I.beta, old[e], acc[e]);
            }
            st_hint<VL>(dst, acc, pol_once);
        }
#pragma unroll
        for (int e = 0; e < VL; ++e) acc[e] = 0.0f;
    };
    auto step = [&](int p, float v, const float (&b)[VL]) {
        while (p >= re) {
            emit(r);
            ++r;
            if (r - rb >= 32) {
                rb += 32;
                rc = rn;
                rn = __ldg(I.rowPtr + min(rb + 33 + lane, I.nr));
            }
            re = __shfl_sync(kFull, rc, r - rb);
        }
#pragma unroll
        for (int e = 0; e < VL; ++e) acc[e] = fmaf(v, b[e], acc[e]);
    };
    auto load_win = [&](int wb, int &cc, float &vv) {
        const bool ok = wb + lane < k1;
        cc = ok ? ld_hint_s32(I.colIdx + wb + lane, pol_once) : 0;
        vv = ok ? ld_val<TV>(Av + wb + lane, pol_once) : 0.0f;
    };
    int ccur, cnext;
    float vcur, vnext;
    load_win(k0, ccur, vcur);
    for (int wb = k0; wb < k1; wb += 32) {
        load_win(wb + 32, cnext, vnext);
        const int cnt = min(32, k1 - wb);
        int t = 0;
        for (; t + U <= cnt; t += U) {
            int cc[U];
            float vv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                cc[u] = __shfl_sync(kFull, ccur, t + u);
                vv[u] = __shfl_sync(kFull, vcur, t + u);
            }
            float b[U][VL];
#pragma unroll
            for (int u = 0; u < U; ++u) ld_b<TB, VL>(b[u], Bl + (size_t)cc[u] * I.ldb);
#pragma unroll
            for (int u = 0; u < U; ++u) step(wb + t + u, vv[u], b[u]);
        }
        for (; t < cnt; ++t) {
            float b[VL];
            ld_b<TB, VL>(b, Bl + (size_t)__shfl_sync(kFull, ccur, t) * I.ldb);
            step(wb + t, __shfl_sync(kFull, vcur, t), b);
        }
        ccur = cnext;
        vcur = vnext;
    }
    while (r < row1) {  // rows ending at k1, trailing empty rows included
        emit(r);
        ++r;
    }
}

template <int W, typename TV, typename TB>
__global__ void __launch_bounds__(256, DASPMM_LEAN_MINB)
    k_batch_spmm(const BatchInst *__restrict__ inst, const BatchItem *__restrict__ items,
                 long long nitems, unsigned long long *head)
{
    const uint64_t pol_once = policy_evict_first();
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long g = 0;
        if (lane == 0) g = atomicAdd(head, 1ull);
        g = __shfl_sync(kFull, g, 0);
        if (g >= (unsigned long long)nitems) return;
        const BatchItem it = items[g];
        const BatchInst I = inst[it.inst];
        batch_rows<W, DASPMM_LEAN_U, TV, TB>(I, it.row0, it.row1, it.ctile * W, pol_once);
    }
}

}  // namespace daspmm

using namespace daspmm;

struct daspmm_batch_s {
    int device = 0;
    int ninst = 0, nv = 0, val_fmt = 0, b_fmt = 0, W = 0, chunk = 0;
    long long nitems = 0, total_nnz = 0;
    BatchInst *d_inst = nullptr;
    long long *d_begin = nullptr;
    BatchItem *d_items = nullptr;
    unsigned long long *d_head = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

template <int W, typename TV, typename TB>
void launch_batch_w(daspmm_batch_s *b, cudaStream_t st)
{
    const unsigned grid = (unsigned)std::max<long long>(
        1, std::min<long long>((long long)device_sms() * DASPMM_LEAN_MINB, (b->nitems + 7) / 8));
    k_batch_spmm<W, TV, TB><<<grid, 256, 0, st>>>(b->d_inst, b->d_items, b->nitems, b->d_head);
}

template <typename TV, typename TB>
void launch_batch_t(daspmm_batch_s *b, cudaStream_t st)
{
    if (b->W == 128) launch_batch_w<128, TV, TB>(b, st);
    else if (b->W == 64) launch_batch_w<64, TV, TB>(b, st);
    else launch_batch_w<32, TV, TB>(b, st);
}

daspmm_status batch_launch(daspmm_batch_s *b, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(b->d_head, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail(e);
    timer_before(st);
    if (b->val_fmt == DASPMM_F32 && b->b_fmt == DASPMM_F32) launch_batch_t<float, float>(b, st);
    else if (b->val_fmt == DASPMM_F32 && b->b_fmt == DASPMM_BF16) launch_batch_t<float, bf16>(b, st);
    else if (b->val_fmt == DASPMM_BF16 && b->b_fmt == DASPMM_BF16) launch_batch_t<bf16, bf16>(b, st);
    else if (b->val_fmt == DASPMM_F32 && b->b_fmt == DASPMM_E4M3) launch_batch_t<float, fp8>(b, st);
    else launch_batch_t<bf16, fp8>(b, st);
    timer_after(st);
    count_launches(1);
    e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

void batch_free(daspmm_batch_s *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_inst);
    cudaFree(b->d_begin);
    cudaFree(b->d_items);
    cudaFree(b->d_head);
    delete b;
}

size_t fmt_size(int f) { return f == DASPMM_F32 ? 4 : (f == DASPMM_E4M3 ? 1 : 2); }

}  // namespace

extern "C" {

daspmm_status daspmm_batch_create(const daspmm_instance *inst, int n, const daspmm_config *cfg,
                                  daspmm_batch *out, void *stream)
{
    if (!out || n < 0 || (n > 0 && !inst)) return DASPMM_ERR_INVALID;
    *out = nullptr;
    daspmm_batch_s *b = new (std::nothrow) daspmm_batch_s;
    if (!b) return DASPMM_ERR_NOMEM;
    cudaStream_t st = (cudaStream_t)stream;
    cudaGetDevice(&b->device);
    b->ninst = n;
    b->chunk = (cfg && cfg->chunk > 0) ? cfg->chunk : 256;
    if (n > 0) {
        b->nv = inst[0].nv;
        b->val_fmt = inst[0].val_fmt;
        b->b_fmt = inst[0].b_fmt;
    }
    const bool combo = (b->val_fmt == DASPMM_F32 && b->b_fmt == DASPMM_F32) ||
                       (b->val_fmt == DASPMM_F32 && b->b_fmt == DASPMM_BF16) ||
                       (b->val_fmt == DASPMM_BF16 && b->b_fmt == DASPMM_BF16) ||
                       (b->val_fmt == DASPMM_F32 && b->b_fmt == DASPMM_E4M3) ||
                       (b->val_fmt == DASPMM_BF16 && b->b_fmt == DASPMM_E4M3);
    if (n > 0 && (!combo || b->nv < 1)) {
        delete b;
        return DASPMM_ERR_UNSUPPORTED;
    }
    // tile width: the widest of 128 / 64 / 32 dividing nv, else 32 (lanes masked)
    const int nv = std::max(1, b->nv);
    b->W = nv % 128 == 0 ? 128 : (nv % 64 == 0 ? 64 : 32);
    const int VL = b->W / 32;
    std::vector<BatchInst> hi(n);
    std::vector<long long> begin(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        const daspmm_instance &s = inst[i];
        if (s.nv != b->nv || s.val_fmt != b->val_fmt || s.b_fmt != b->b_fmt || s.nr < 0 ||
            s.nc < 0 || s.nnz < 0 || s.nv % VL != 0 || (s.nr > 0 && (!s.rowPtr || !s.C)) ||
            (s.nnz > 0 && (!s.colIdx || !s.values || !s.B)) ||
            (s.b_fmt == DASPMM_E4M3 && !s.b_scales) ||
            ((uintptr_t)s.B % (VL * fmt_size(s.b_fmt))) || ((uintptr_t)s.C % (VL * 4))) {
            delete b;
            return DASPMM_ERR_INVALID;
        }
        BatchInst &d = hi[i];
        d.nr = s.nr; d.nc = s.nc; d.nnz = s.nnz; d.nv = s.nv;
        d.ldb = s.nv; d.ldc = s.nv;
        d.row_tiles = s.nr == 0 ? 0 : (int)std::max<long long>(1, ((long long)s.nnz + b->chunk - 1) / b->chunk);
        d.col_tiles = (s.nv + b->W - 1) / b->W;
        d.rowPtr = s.rowPtr; d.colIdx = s.colIdx; d.vals = s.values; d.B = s.B;
        d.bscale = s.b_scales; d.C = s.C; d.beta = s.beta;
        begin[i + 1] = begin[i] + (long long)d.row_tiles * d.col_tiles;
        b->total_nnz += s.nnz;
    }
    b->nitems = begin[n];
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&b->d_head, sizeof(unsigned long long));
    if (e == cudaSuccess && n) e = cudaMalloc(&b->d_inst, sizeof(BatchInst) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_begin, sizeof(long long) * (n + 1));
    if (e == cudaSuccess && b->nitems) e = cudaMalloc(&b->d_items, sizeof(BatchItem) * b->nitems);
    if (e != cudaSuccess) {
        cudaGetLastError();
        batch_free(b);
        return DASPMM_ERR_NOMEM;
    }
    if (n) e = cudaMemcpyAsync(b->d_inst, hi.data(), sizeof(BatchInst) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_begin, begin.data(), sizeof(long long) * (n + 1),
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && b->nitems) {
        const unsigned g = (unsigned)((b->nitems + 255) / 256);
        k_batch_plan<<<g, 256, 0, st>>>(b->d_inst, b->d_begin, n, b->chunk, b->d_items, b->nitems);
        count_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host vectors go out of scope
    if (e != cudaSuccess) {
        batch_free(b);
        return cuda_fail(e);
    }
    *out = b;
    return DASPMM_OK;
}

daspmm_status daspmm_batch_run(daspmm_batch b, void *stream)
{
    if (!b) return DASPMM_ERR_INVALID;
    if (b->nitems == 0) return DASPMM_OK;
    return batch_launch(b, (cudaStream_t)stream);
}

daspmm_status daspmm_batch_capture(daspmm_batch b, void *stream)
{
    if (!b) return DASPMM_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    if (!st) return DASPMM_ERR_INVALID;  // the legacy stream cannot be captured
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(e);
    daspmm_status s = b->nitems ? batch_launch(b, st) : DASPMM_OK;
    e = cudaStreamEndCapture(st, &b->graph);
    if (s != DASPMM_OK) return s;
    if (e != cudaSuccess) return cuda_fail(e);
    e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

daspmm_status daspmm_batch_replay(daspmm_batch b, void *stream)
{
    if (!b || !b->exec) return DASPMM_ERR_INVALID;
    cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    if (e == cudaSuccess) count_launches(b->nitems ? 1 : 0);
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

daspmm_status daspmm_batch_info(daspmm_batch b, long long *nitems, long long *total_nnz)
{
    if (!b) return DASPMM_ERR_INVALID;
    if (nitems) *nitems = b->nitems;
    if (total_nnz) *total_nnz = b->total_nnz;
    return DASPMM_OK;
}

daspmm_status daspmm_batch_tune(const daspmm_instance *inst, int n, const int *chunks,
                                int nchunks, int reps, int *best_chunk, float *best_us,
                                void *stream)
{
    static const int kDefault[] = {128, 256, 512, 1024};
    if (!chunks || nchunks <= 0) {
        chunks = kDefault;
        nchunks = 4;
    }
    if (!best_chunk || reps < 0) return DASPMM_ERR_INVALID;
    if (reps == 0) reps = 5;
    cudaStream_t st = (cudaStream_t)stream;
    float bus = 0.0f;
    int bch = 0;
    for (int k = 0; k < nchunks; ++k) {
        daspmm_config cfg{};
        cfg.chunk = chunks[k];
        daspmm_batch b = nullptr;
        daspmm_status s = daspmm_batch_create(inst, n, &cfg, &b, stream);
        if (s != DASPMM_OK) return s;
        for (int i = 0; i < 2 && s == DASPMM_OK; ++i) s = daspmm_batch_run(b, stream);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, st);
        for (int i = 0; i < reps && s == DASPMM_OK; ++i) s = daspmm_batch_run(b, stream);
        cudaEventRecord(e1, st);
        float ms = 0.0f;
        cudaError_t e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        daspmm_batch_destroy(b);
        if (s != DASPMM_OK) return s;
        if (e != cudaSuccess) return cuda_fail(e);
        const float us = ms * 1000.0f / reps;
        if (bch == 0 || us < bus) {
            bus = us;
            bch = chunks[k];
        }
    }
    *best_chunk = bch;
    if (best_us) *best_us = bus;
    return DASPMM_OK;
}

daspmm_status daspmm_batch_destroy(daspmm_batch b)
{
    if (!b) return DASPMM_OK;
    batch_free(b);
    return DASPMM_OK;
}

}  // extern "C"
