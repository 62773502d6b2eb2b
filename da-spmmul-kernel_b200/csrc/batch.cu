// batch.cu -- many SpMMs of uneven sizes in one persistent launch.
//
// The reference runs one problem per cudaSpmm call (spmvspmm.h:53-199); a
// batch here is a table of instances (each its own CSR A, dense B and C and
// column count nv; all with the same storage formats).  Every matrix is cut
// once into tiles of about `chunk` nonzeros (build_tiles): runs of whole rows,
// and pieces of rows longer than `chunk`, so no work item is longer than one
// chunk whatever the row-length distribution.  A plan kernel lists the work
// items -- (instance, tile, column tile) -- and the persistent kernel's warps
// take them from a device queue (one atomic per item).  A run of rows is
// gathered like the lean balanced kernel (windows of 32 nonzeros, four B rows
// in flight, row ends from a lane cache); a piece stores its partial sum in a
// slot and the row's last piece to finish adds the slots in piece order.
// A result therefore depends only on its own instance (matrix, nv, chunk),
// never on the rest of the batch or on scheduling.
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

// item g -> (instance, tile, column tile).
static __global__ void k_batch_plan(const BatchInst *__restrict__ inst,
                                    const long long *__restrict__ item_begin, int ninst,
                                    BatchItem *items, long long nitems)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nitems) return;
    int lo = 0, hi = ninst;  // last i with item_begin[i] <= g
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (item_begin[mid] <= g) lo = mid;
        else hi = mid;
    }
    const int ct_n = inst[lo].col_tiles;
    const long long local = g - item_begin[lo];
    BatchItem it;
    it.inst = lo;
    it.tile = (int)(local / ct_n);
    it.ctile = (int)(local % ct_n);
    it.pad_ = 0;
    items[g] = it;
}

// Rows [row0, row1) of one instance, column tile [tb0, tb0 + W): the lean
// windowed gather over whole rows (no carries).  Lanes whose columns lie at or
// past nv (nv % W != 0) load a clamped, in-bounds vector and store nothing.
template <int W, int U, typename TV, typename TB>
__device__ __noinline__ void batch_rows(const BatchInst &I, int row0, int row1, int tb0,
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

// Rows [row0, row1) of one instance, none of them empty, beta == 0: the ends
// of the rows finishing in a window of 32 nonzeros come as one bitmask (lane l
// looks at the end of row r + l; with no empty row the 32 lanes cover every
// row that can end in the window), so the window is summed straight through
// and a row is stored at its bit.  Same sums, in the same order, as
// batch_rows.
template <int W, int U, typename TV, typename TB>
__device__ __forceinline__ void batch_rows_fast(const BatchInst &I, int row0, int row1,
                                                int tb0, uint64_t pol_once)
{
    constexpr int VL = W / 32;
    constexpr bool SCALED = std::is_same<TB, fp8>::value;
    const int lane = threadIdx.x & 31;
    const int col = tb0 + lane * VL;
    const bool active = col < I.nv;
    const int colc = active ? col : I.nv - VL;  // nv % VL == 0 (checked on the host)
    const TB *Bl = reinterpret_cast<const TB *>(I.B) + colc;
    const TV *Av = reinterpret_cast<const TV *>(I.vals);
    const int k0 = __ldg(I.rowPtr + row0), k1 = __ldg(I.rowPtr + row1);
    int r = row0;
    int E = __ldg(I.rowPtr + min(r + 1 + lane, I.nr));
    float acc[VL];
#pragma unroll
    for (int e = 0; e < VL; ++e) acc[e] = 0.0f;
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
        const int pos = E - 1 - wb;
        const bool in = r + lane < row1 && pos >= 0 && pos < cnt;
        const unsigned ends = __reduce_or_sync(kFull, in ? (1u << pos) : 0u);
        E = __ldg(I.rowPtr + min(r + __popc(ends) + 1 + lane, I.nr));  // next window's
        float *cdst = I.C + (size_t)r * I.ldc + col;
#pragma unroll
        for (int g = 0; g < 32 / U; ++g) {
            int cc[U];
            float vv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                cc[u] = __shfl_sync(kFull, ccur, g * U + u);
                vv[u] = __shfl_sync(kFull, vcur, g * U + u);
            }
            float b[U][VL];
#pragma unroll
            for (int u = 0; u < U; ++u) ld_b<TB, VL>(b[u], Bl + (size_t)cc[u] * I.ldb);
#pragma unroll
            for (int u = 0; u < U; ++u) {
#pragma unroll
                for (int e = 0; e < VL; ++e) acc[e] = fmaf(vv[u], b[u][e], acc[e]);
                if ((ends >> (g * U + u)) & 1u) {
                    if (active) {
                        if constexpr (SCALED) {
#pragma unroll
                            for (int e = 0; e < VL; ++e) acc[e] *= __ldg(I.bscale + col + e);
                        }
                        st_hint<VL>(cdst, acc, pol_once);
                    }
#pragma unroll
                    for (int e = 0; e < VL; ++e) acc[e] = 0.0f;
                    ++r;
                    cdst += I.ldc;
                }
            }
        }
        ccur = cnext;
        vcur = vnext;
    }
}

// One piece (nonzeros [k0, k1) of row row0) for column tile [tb0, tb0 + W):
// the partial sum goes to the piece's slot; the row's last piece to arrive
// adds all slots in piece order, scales, applies beta and stores the row.
template <int W, int U, typename TV, typename TB>
__device__ __noinline__ void batch_piece(const BatchInst &I, const BatchTile &T, int ct,
                                            uint64_t pol_once)
{
    constexpr int VL = W / 32;
    constexpr bool SCALED = std::is_same<TB, fp8>::value;
    const int lane = threadIdx.x & 31;
    const int col = ct * W + lane * VL;
    const bool active = col < I.nv;
    const int colc = active ? col : I.nv - VL;
    const TB *Bl = reinterpret_cast<const TB *>(I.B) + colc;
    const TV *Av = reinterpret_cast<const TV *>(I.vals);
    float acc[VL];
#pragma unroll
    for (int e = 0; e < VL; ++e) acc[e] = 0.0f;
    for (int wb = T.k0; wb < T.k1; wb += 32) {
        const bool ok = wb + lane < T.k1;
        const int cl = ok ? ld_hint_s32(I.colIdx + wb + lane, pol_once) : 0;
        const float vl = ok ? ld_val<TV>(Av + wb + lane, pol_once) : 0.0f;
        const int cnt = min(32, T.k1 - wb);
        int t = 0;
        for (; t + U <= cnt; t += U) {
            float b[U][VL];
#pragma unroll
            for (int u = 0; u < U; ++u)
                ld_b<TB, VL>(b[u], Bl + (size_t)__shfl_sync(kFull, cl, t + u) * I.ldb);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const float v = __shfl_sync(kFull, vl, t + u);
#pragma unroll
                for (int e = 0; e < VL; ++e) acc[e] = fmaf(v, b[u][e], acc[e]);
            }
        }
        for (; t < cnt; ++t) {
            float b[VL];
            ld_b<TB, VL>(b, Bl + (size_t)__shfl_sync(kFull, cl, t) * I.ldb);
            const float v = __shfl_sync(kFull, vl, t);
#pragma unroll
            for (int e = 0; e < VL; ++e) acc[e] = fmaf(v, b[e], acc[e]);
        }
    }
    float part[VL];
#pragma unroll
    for (int e = 0; e < VL; ++e) part[e] = acc[e];
    float *slot0 = I.slots + (size_t)T.slot * I.nv + col;
    if (active) st_v<VL>(slot0 + (size_t)T.piece * I.nv, part);
    __threadfence();
    __syncwarp();
    int *counter = I.cnt + (size_t)T.cnt * I.col_tiles + ct;
    int last = 0;
    if (lane == 0) last = atomicAdd(counter, 1) == T.npieces - 1;
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    __threadfence();
    if (lane == 0) *counter = 0;  // every piece has arrived: ready for the next run
    if (!active) return;
    float tot[VL];
#pragma unroll
    for (int e = 0; e < VL; ++e) tot[e] = 0.0f;
    for (int p = 0; p < T.npieces; ++p) {
        float h[VL];
        if (p == T.piece) {
#pragma unroll
            for (int e = 0; e < VL; ++e) h[e] = part[e];
        } else {
            ld_cg<VL>(h, slot0 + (size_t)p * I.nv);
        }
#pragma unroll
        for (int e = 0; e < VL; ++e) tot[e] += h[e];
    }
    float *dst = I.C + (size_t)T.row0 * I.ldc + col;
#pragma unroll
    for (int e = 0; e < VL; ++e) tot[e] *= SCALED ? __ldg(I.bscale + col + e) : 1.0f;
    if (I.beta != 0.0f) {
        float old[VL];
        ld_plain<VL>(old, dst);
#pragma unroll
        for (int e = 0; e < VL; ++e) tot[e] = fmaf(I.beta, old[e], tot[e]);
    }
    st_v<VL>(dst, tot);
}

#ifndef DASPMM_BATCH_U16
#define DASPMM_BATCH_U16 8  // B rows in flight per warp step for 2- and 1-byte B
#endif

template <int W, typename TV, typename TB>
__device__ __forceinline__ void batch_item(const BatchInst &I, const BatchTile &T, int ct,
                                           uint64_t pol_once)
{
    // a lane's share of a B row in 2- or 1-byte storage is a few bytes: more
    // rows in flight per step keep the warp's bytes in flight up (measured on
    // the 512-instance BF16 batch, N = 64: U = 4 3.03 ms, 8 2.90 ms, 16 3.37 ms)
    constexpr int UF = sizeof(TB) < 4 ? DASPMM_BATCH_U16 : DASPMM_LEAN_U;
    if (T.piece >= 0)
        batch_piece<W, DASPMM_LEAN_U, TV, TB>(I, T, ct, pol_once);
    else if (T.npieces == 0 && I.beta == 0.0f)  // a run without empty rows
        batch_rows_fast<W, UF, TV, TB>(I, T.row0, T.row1, ct * W, pol_once);
    else
        batch_rows<W, DASPMM_LEAN_U, TV, TB>(I, T.row0, T.row1, ct * W, pol_once);
}

#ifndef DASPMM_BATCH_MINB
#define DASPMM_BATCH_MINB DASPMM_LEAN_MINB  // CTAs of 256 threads per SM
#endif
#ifndef DASPMM_BATCH_GRP
#define DASPMM_BATCH_GRP 1  // runs of rows and pieces take the worker-group gather
#endif

// WM: the tile width every instance uses, or 0 for a batch of mixed widths
// (a warp-uniform switch on the item's instance).
template <int WM, typename TV, typename TB>
__global__ void __launch_bounds__(256, DASPMM_BATCH_MINB)
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
        const BatchInst &I = inst[it.inst];  // fields read on use (L1-resident)
        const BatchTile T = I.tiles[it.tile];
        if constexpr (WM != 0) {
            batch_item<WM, TV, TB>(I, T, it.ctile, pol_once);
        } else {
            if (I.W == 128) batch_item<128, TV, TB>(I, T, it.ctile, pol_once);
            else if (I.W == 64) batch_item<64, TV, TB>(I, T, it.ctile, pol_once);
            else batch_item<32, TV, TB>(I, T, it.ctile, pol_once);
        }
    }
}

// One item of instance *I, column tile ct, for the G lanes of this worker
// (one of the warp's 32 / G workers, each on its own item, all in step),
// gathered like the single-product group kernel: windows of G nonzeros, one
// lane load of EPL elements per lane and row, UU rows in flight.  A run of
// whole rows without empty rows (beta == 0) stores each row at its bit of the
// window's row-end mask; a piece of a long row sums its nonzeros, leaves the
// partial in its slot and, if it is the row's last piece to arrive, adds the
// slots in piece order and stores the row.  The same FMAs and additions in
// the same order as batch_rows_fast and batch_piece, so an item gives the
// same bits on either path.  Positions past the worker's last nonzero load
// nothing and add an exact zero.
template <int G, int EPL, int U, typename TV, typename TB>
__device__ __forceinline__ void batch_item_grp(const BatchInst *__restrict__ I,
                                               const BatchTile &T, int ct, bool have,
                                               uint64_t pol_once)
{
    constexpr int RAW = EPL * (int)sizeof(TB) / 4;  // 32-bit words per lane load
    constexpr int UU = U < G ? U : G;
    constexpr unsigned GM = G == 32 ? 0xFFFFFFFFu : ((1u << G) - 1u);
    constexpr bool SCALED = std::is_same<TB, fp8>::value;
    const int lane = threadIdx.x & 31, w = lane / G, gl = lane % G;
    const unsigned gmask = GM << (G * w);
    const int col = ct * (G * EPL) + gl * EPL;
    const bool piece = have && T.piece >= 0;
    const int *rp = have ? I->rowPtr : nullptr;
    const int *ci = have ? I->colIdx : nullptr;
    const TV *Av = have ? reinterpret_cast<const TV *>(I->vals) : nullptr;
    const TB *Bl = have ? reinterpret_cast<const TB *>(I->B) + col : nullptr;
    const int ldb = have ? I->ldb : 0, ldc = have ? I->ldc : 0, nr = have ? I->nr : 0;
    const int row1 = have ? T.row1 : 0;
    const int k0 = !have ? 0 : (piece ? T.k0 : __ldg(rp + T.row0));
    const int k1 = !have ? 0 : (piece ? T.k1 : __ldg(rp + T.row1));
    int r = have ? T.row0 : 0;
    int E = (have && !piece) ? __ldg(rp + min(r + 1 + gl, nr)) : 0;
    int nwin = (k1 - k0 + G - 1) / G;
#pragma unroll
    for (int o = G; o < 32; o <<= 1) nwin = max(nwin, __shfl_xor_sync(kFull, nwin, o));
    float acc[EPL];
#pragma unroll
    for (int e = 0; e < EPL; ++e) acc[e] = 0.0f;
    auto load_win = [&](int wb, int &c, float &v) {
        const bool ok = wb + gl < k1;
        c = ok ? ld_hint_s32(ci + wb + gl, pol_once) : 0;
        v = ok ? ld_val<TV>(Av + wb + gl, pol_once) : 0.0f;
    };
    int ccur, cnext;
    float vcur, vnext;
    int wb = k0;
    load_win(wb, ccur, vcur);
    for (int wi = 0; wi < nwin; ++wi, wb += G) {
        load_win(wb + G, cnext, vnext);
        const int cnt = k1 - wb;  // nonzeros of this worker left (<= 0: none)
        const int pos = E - 1 - wb;
        const bool in = have && !piece && r + gl < row1 && pos >= 0 && pos < min(cnt, G);
        const unsigned e32 = __reduce_or_sync(kFull, in ? (1u << (pos + G * w)) : 0u);
        const unsigned ends = (e32 >> (G * w)) & GM;
        if (have && !piece) E = __ldg(rp + min(r + __popc(ends) + 1 + gl, nr));  // next window's
        float *cdst = (have && !piece) ? I->C + (size_t)r * ldc + col : nullptr;
#pragma unroll
        for (int g = 0; g < G / UU; ++g) {
            int cc[UU];
            float vv[UU];
#pragma unroll
            for (int u = 0; u < UU; ++u) {
                cc[u] = __shfl_sync(kFull, ccur, g * UU + u, G);
                vv[u] = __shfl_sync(kFull, vcur, g * UU + u, G);
            }
            uint32_t b[UU][RAW];
#pragma unroll
            for (int u = 0; u < UU; ++u) {
                if (g * UU + u < cnt) {
                    ld_raw<RAW>(b[u], Bl + (size_t)cc[u] * ldb);
                } else {
#pragma unroll
                    for (int i = 0; i < RAW; ++i) b[u][i] = 0u;
                }
            }
#pragma unroll
            for (int u = 0; u < UU; ++u) {
#pragma unroll
                for (int e = 0; e < EPL; ++e)
                    acc[e] = fmaf(vv[u], elem<TB, RAW>(b[u], e), acc[e]);
                if ((ends >> (g * UU + u)) & 1u) {
                    if constexpr (SCALED) {
#pragma unroll
                        for (int e = 0; e < EPL; ++e) acc[e] *= __ldg(I->bscale + col + e);
                    }
                    st_hint_n<EPL>(cdst, acc, pol_once);
#pragma unroll
                    for (int e = 0; e < EPL; ++e) acc[e] = 0.0f;
                    ++r;
                    cdst += ldc;
                }
            }
            asm volatile("" ::: "memory");
        }
        ccur = cnext;
        vcur = vnext;
    }
    if (!piece) return;
    // the piece's partial, then the row's last piece adds all of them
    const int nv = I->nv;
    float *slot0 = I->slots + (size_t)T.slot * nv + col;
    st_n<EPL>(slot0 + (size_t)T.piece * nv, acc);
    __threadfence();
    __syncwarp(gmask);
    int *counter = I->cnt + (size_t)T.cnt * I->col_tiles + ct;
    int last = 0;
    if (gl == 0) last = atomicAdd(counter, 1) == T.npieces - 1;
    last = __shfl_sync(gmask, last, 0, G);
    if (!last) return;
    __threadfence();
    if (gl == 0) *counter = 0;  // every piece has arrived: ready for the next run
    float tot[EPL];
#pragma unroll
    for (int e = 0; e < EPL; ++e) tot[e] = 0.0f;
    for (int p = 0; p < T.npieces; ++p) {
        float h[EPL];
        if (p == T.piece) {
#pragma unroll
            for (int e = 0; e < EPL; ++e) h[e] = acc[e];
        } else {
            ld_cg_n<EPL>(h, slot0 + (size_t)p * nv);
        }
#pragma unroll
        for (int e = 0; e < EPL; ++e) tot[e] += h[e];
    }
    if constexpr (SCALED) {
#pragma unroll
        for (int e = 0; e < EPL; ++e) tot[e] *= __ldg(I->bscale + col + e);
    }
    st_n<EPL>(I->C + (size_t)T.row0 * ldc + col, tot);
}

// The persistent batch kernel with G-lane workers: a warp claims 32 / G
// consecutive items; the runs without empty rows and the pieces of long rows
// (beta == 0, tile width WG, 32-byte aligned B, C and slots) are gathered
// together by batch_item_grp, every other item (runs with empty rows, other
// widths) by the whole warp with batch_item after it.
template <int WG, int G, int EPL, int U, typename TV, typename TB, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_batch_grp(const BatchInst *__restrict__ inst, const BatchItem *__restrict__ items,
                long long nitems, unsigned long long *head)
{
    static_assert(G * EPL == WG, "a worker covers one column tile");
    constexpr int NW = 32 / G;
    const uint64_t pol_once = policy_evict_first();
    const int lane = threadIdx.x & 31, w = lane / G;
    for (;;) {
        unsigned long long g0 = 0;
        if (lane == 0) g0 = atomicAdd(head, (unsigned long long)NW);
        g0 = __shfl_sync(kFull, g0, 0);
        if (g0 >= (unsigned long long)nitems) return;
        const long long gi = (long long)g0 + w;
        const bool valid = gi < nitems;
        BatchItem it{};
        const BatchInst *I = nullptr;
        BatchTile T{};
        if (valid) {
            it = items[gi];
            I = inst + it.inst;
            T = I->tiles[it.tile];
        }
        const bool fast = valid && I->grp && I->W == WG && I->beta == 0.0f &&
                          (T.piece >= 0 ? (reinterpret_cast<uintptr_t>(I->slots) & 31) == 0
                                        : T.npieces == 0);
        if (__any_sync(kFull, fast))
            batch_item_grp<G, EPL, U, TV, TB>(I, T, it.ctile, fast, pol_once);
        unsigned slow = __ballot_sync(kFull, valid && !fast && lane % G == 0);
        while (slow) {  // warp-uniform
            const int l = __ffs(slow) - 1;
            slow &= slow - 1;
            const BatchItem it2 = items[(long long)g0 + l / G];
            const BatchInst &I2 = inst[it2.inst];
            const BatchTile T2 = I2.tiles[it2.tile];
            if (I2.W == 128) batch_item<128, TV, TB>(I2, T2, it2.ctile, pol_once);
            else if (I2.W == 64) batch_item<64, TV, TB>(I2, T2, it2.ctile, pol_once);
            else batch_item<32, TV, TB>(I2, T2, it2.ctile, pol_once);
        }
    }
}

template <int WG, int G, int EPL, int U, typename TV, typename TB, int MINB>
void launch_batch_grp(const BatchInst *d_inst, const BatchItem *d_items, long long nitems,
                      unsigned long long *d_head, cudaStream_t st)
{
    const long long claims = (nitems + 32 / G - 1) / (32 / G);
    const unsigned grid = (unsigned)std::max<long long>(
        1, std::min<long long>((long long)device_sms() * MINB, (claims + 7) / 8));
    k_batch_grp<WG, G, EPL, U, TV, TB, MINB><<<grid, 256, 0, st>>>(d_inst, d_items, nitems,
                                                                   d_head);
}

// Worker shapes for the group gather, measured on the 512-instance batch with
// tiles sorted by size (ms, best row tile; the 32-lane kernel in brackets).
// FP32 B: 32-byte lane loads for 128- and 64-column tiles, 16-byte for 32
// (N = 32 / 64 / 128: 1.73 / 2.50 / 4.54 [2.70 / 3.19 / 4.86]).  BF16 B:
// 16-byte loads in 8-lane workers for 64 columns, 32-byte for 128, 8-byte
// for 32 (FP32 values: 1.64 / 2.20 / 3.39 [2.50 / 2.89 / 3.99]; BF16 values
// 1.66 / 2.25 / 3.63 [2.50 / 2.87 / 3.88]).  E4M3 B: 8-byte loads for 64 and
// 32 columns (1.69 / 2.31 [2.65 / 2.95]); at 128 columns the group form only
// ties (3.93 [3.92]; 4.31 with tiles in row order), so it keeps the 32-lane
// kernel there.
template <typename TV, typename TB>
bool launch_batch_grp_t(int wg, const BatchInst *d_inst, const BatchItem *d_items,
                        long long nitems, unsigned long long *d_head, cudaStream_t st)
{
    if constexpr (std::is_same<TB, float>::value) {
        if (wg == 128) launch_batch_grp<128, 16, 8, 8, TV, TB, 2>(d_inst, d_items, nitems, d_head, st);
        else if (wg == 64) launch_batch_grp<64, 8, 8, 8, TV, TB, 2>(d_inst, d_items, nitems, d_head, st);
        else if (wg == 32) launch_batch_grp<32, 8, 4, 8, TV, TB, 3>(d_inst, d_items, nitems, d_head, st);
        else return false;
    } else if constexpr (sizeof(TB) == 2) {
        if (wg == 128) launch_batch_grp<128, 8, 16, 8, TV, TB, 2>(d_inst, d_items, nitems, d_head, st);
        else if (wg == 64) launch_batch_grp<64, 8, 8, 16, TV, TB, 3>(d_inst, d_items, nitems, d_head, st);
        else if (wg == 32) launch_batch_grp<32, 8, 4, 16, TV, TB, 3>(d_inst, d_items, nitems, d_head, st);
        else return false;
    } else {
        if (wg == 64) launch_batch_grp<64, 8, 8, 16, TV, TB, 3>(d_inst, d_items, nitems, d_head, st);
        else if (wg == 32) launch_batch_grp<32, 4, 8, 16, TV, TB, 3>(d_inst, d_items, nitems, d_head, st);
        else return false;
    }
    return true;
}

size_t fmt_size(int f) { return f == DASPMM_F32 ? 4 : (f == DASPMM_E4M3 ? 1 : 2); }

template <int WM, typename TV, typename TB>
void launch_batch_w(const BatchInst *d_inst, const BatchItem *d_items, long long nitems,
                    unsigned long long *d_head, cudaStream_t st)
{
    const unsigned grid = (unsigned)std::max<long long>(
        1, std::min<long long>((long long)device_sms() * DASPMM_BATCH_MINB, (nitems + 7) / 8));
    k_batch_spmm<WM, TV, TB><<<grid, 256, 0, st>>>(d_inst, d_items, nitems, d_head);
}

// grp: every instance shares the tile width wmode and qualifies for the
// worker-group gather (BatchInst::grp); the group kernel then takes the batch.
// Otherwise the 32-lane kernel: in the group kernel, items it cannot gather
// run the 32-lane code one after another at its lower occupancy (on the
// 64-matrix serving pool, mixed widths: capacity 56.6k against 66.5k req/s).
template <typename TV, typename TB>
void launch_batch_t(int wmode, bool grp, const BatchInst *d_inst, const BatchItem *d_items,
                    long long nitems, unsigned long long *d_head, cudaStream_t st)
{
    if (DASPMM_BATCH_GRP && grp &&
        launch_batch_grp_t<TV, TB>(wmode, d_inst, d_items, nitems, d_head, st))
        return;
    if (wmode == 128) launch_batch_w<128, TV, TB>(d_inst, d_items, nitems, d_head, st);
    else if (wmode == 64) launch_batch_w<64, TV, TB>(d_inst, d_items, nitems, d_head, st);
    else if (wmode == 32) launch_batch_w<32, TV, TB>(d_inst, d_items, nitems, d_head, st);
    else launch_batch_w<0, TV, TB>(d_inst, d_items, nitems, d_head, st);
}

int batch_tile_width(int nv) { return nv % 128 == 0 ? 128 : (nv % 64 == 0 ? 64 : 32); }

bool batch_formats_ok(int vf, int bf)
{
    return (vf == DASPMM_F32 && bf == DASPMM_F32) || (vf == DASPMM_F32 && bf == DASPMM_BF16) ||
           (vf == DASPMM_BF16 && bf == DASPMM_BF16) || (vf == DASPMM_F32 && bf == DASPMM_E4M3) ||
           (vf == DASPMM_BF16 && bf == DASPMM_E4M3);
}

daspmm_status batch_fill(const daspmm_instance &s, BatchInst *d, int wcap)
{
    if (s.nv < 1 || s.nr < 0 || s.nc < 0 || s.nnz < 0) return DASPMM_ERR_INVALID;
    int W = batch_tile_width(s.nv);
    if (wcap == 32 || wcap == 64) W = std::min(W, wcap);  // narrower column tiles
    const int VL = W / 32;
    if (s.nv % VL != 0 || (s.nr > 0 && (!s.rowPtr || !s.C)) ||
        (s.nnz > 0 && (!s.colIdx || !s.values || !s.B)) ||
        (s.b_fmt == DASPMM_E4M3 && s.nr > 0 && !s.b_scales) ||
        ((uintptr_t)s.B % (VL * fmt_size(s.b_fmt))) || ((uintptr_t)s.C % (VL * 4)))
        return DASPMM_ERR_INVALID;
    *d = BatchInst{};
    d->nr = s.nr; d->nc = s.nc; d->nnz = s.nnz; d->nv = s.nv;
    d->ldb = s.nv; d->ldc = s.nv;
    d->W = W;
    d->grp = s.nv % W == 0 && (uintptr_t)s.B % 32 == 0 && (uintptr_t)s.C % 32 == 0;
    d->col_tiles = (s.nv + W - 1) / W;
    d->rowPtr = s.rowPtr; d->colIdx = s.colIdx; d->vals = s.values; d->B = s.B;
    d->bscale = s.b_scales; d->C = s.C; d->beta = s.beta;
    return DASPMM_OK;
}

void build_tiles(const int *rp, int nr, int chunk, TilePlan *out)
{
    out->tiles.clear();
    out->npieces = 0;
    out->nlong = 0;
    int r = 0;
    while (r < nr) {
        const int len = rp[r + 1] - rp[r];
        if (len > chunk) {  // a long row: pieces of `chunk` nonzeros
            const int P = (len + chunk - 1) / chunk;
            for (int p = 0; p < P; ++p) {
                BatchTile t;
                t.row0 = r;
                t.row1 = r + 1;
                t.k0 = rp[r] + p * chunk;
                t.k1 = std::min(rp[r + 1], t.k0 + chunk);
                t.piece = p;
                t.npieces = P;
                t.slot = out->npieces;
                t.cnt = out->nlong;
                out->tiles.push_back(t);
            }
            out->npieces += P;
            ++out->nlong;
            ++r;
            continue;
        }
        // a run of short rows: nonzeros + rows (each row costs a store) <= chunk
        BatchTile t{};
        t.row0 = r;
        t.piece = -1;
        long long cost = 0;
        while (r < nr) {
            const int l = rp[r + 1] - rp[r];
            if (l > chunk || (r > t.row0 && cost + l + 1 > chunk)) break;
            cost += l + 1;
            ++r;
        }
        t.row1 = r;
        t.k0 = rp[t.row0];
        t.k1 = rp[r];
        t.npieces = 0;  // a run: its number of empty rows
        for (int q = t.row0; q < r; ++q) t.npieces += rp[q + 1] == rp[q];
        out->tiles.push_back(t);
    }
    // Longest tiles first, tiles of about the same size next to each other:
    // the worker-group batch kernel gathers 32 / G consecutive items in step,
    // to the longest of them (in row order 16 % of its window steps waited on
    // a longer neighbour on the 512-instance batch), and any queue ends
    // better with its short items last.  A tile's result does not depend on
    // its place in the order.
    std::stable_sort(out->tiles.begin(), out->tiles.end(),
                     [](const BatchTile &x, const BatchTile &y) {
                         return x.k1 - x.k0 > y.k1 - y.k0;
                     });
}

daspmm_status batch_plan_async(const BatchInst *d_inst, const long long *d_begin, int n,
                               BatchItem *d_items, long long nitems, cudaStream_t st)
{
    if (nitems <= 0) return DASPMM_OK;
    const unsigned g = (unsigned)((nitems + 255) / 256);
    k_batch_plan<<<g, 256, 0, st>>>(d_inst, d_begin, n, d_items, nitems);
    count_launches(1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

daspmm_status batch_kernel_async(int vf, int bf, int wmode, bool grp, const BatchInst *d_inst,
                                 const BatchItem *d_items, long long nitems,
                                 unsigned long long *d_head, cudaStream_t st)
{
    if (nitems <= 0) return DASPMM_OK;
    cudaError_t e = cudaMemsetAsync(d_head, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail(e);
    timer_before(st);
    if (vf == DASPMM_F32 && bf == DASPMM_F32)
        launch_batch_t<float, float>(wmode, grp, d_inst, d_items, nitems, d_head, st);
    else if (vf == DASPMM_F32 && bf == DASPMM_BF16)
        launch_batch_t<float, bf16>(wmode, grp, d_inst, d_items, nitems, d_head, st);
    else if (vf == DASPMM_BF16 && bf == DASPMM_BF16)
        launch_batch_t<bf16, bf16>(wmode, grp, d_inst, d_items, nitems, d_head, st);
    else if (vf == DASPMM_F32 && bf == DASPMM_E4M3)
        launch_batch_t<float, fp8>(wmode, grp, d_inst, d_items, nitems, d_head, st);
    else
        launch_batch_t<bf16, fp8>(wmode, grp, d_inst, d_items, nitems, d_head, st);
    timer_after(st);
    count_launches(1);
    e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

}  // namespace daspmm

using namespace daspmm;

struct daspmm_batch_s {
    int device = 0;
    int ninst = 0, nv = 0, val_fmt = 0, b_fmt = 0, W = 0, chunk = 0;
    bool grp = true;  // every instance qualifies for the worker-group gather
    long long nitems = 0, total_nnz = 0;
    BatchInst *d_inst = nullptr;
    long long *d_begin = nullptr;
    BatchItem *d_items = nullptr;
    BatchTile *d_tiles = nullptr;
    float *d_slots = nullptr;
    int *d_cnt = nullptr;
    unsigned long long *d_head = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

daspmm_status batch_launch(daspmm_batch_s *b, cudaStream_t st)
{
    return batch_kernel_async(b->val_fmt, b->b_fmt, b->W, b->grp, b->d_inst, b->d_items,
                              b->nitems, b->d_head, st);
}

void batch_free(daspmm_batch_s *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_inst);
    cudaFree(b->d_begin);
    cudaFree(b->d_items);
    cudaFree(b->d_tiles);
    cudaFree(b->d_slots);
    cudaFree(b->d_cnt);
    cudaFree(b->d_head);
    delete b;
}

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
    // lanes_col 16 / 8: column tiles of at most 64 / 32 floats (0, 32: the
    // widest of 128 / 64 / 32 dividing the instance's nv)
    const int wcap = (cfg && (cfg->lanes_col == 8 || cfg->lanes_col == 16)) ? 4 * cfg->lanes_col : 0;
    if (cfg && cfg->lanes_col && cfg->lanes_col != 8 && cfg->lanes_col != 16 && cfg->lanes_col != 32) {
        delete b;
        return DASPMM_ERR_INVALID;
    }
    if (n > 0) {
        b->nv = inst[0].nv;
        b->val_fmt = inst[0].val_fmt;
        b->b_fmt = inst[0].b_fmt;
    }
    if (n > 0 && !batch_formats_ok(b->val_fmt, b->b_fmt)) {
        delete b;
        return DASPMM_ERR_UNSUPPORTED;
    }
    std::vector<BatchInst> hi(n);
    for (int i = 0; i < n; ++i) {
        const daspmm_instance &s = inst[i];
        const daspmm_status fs = (s.val_fmt != b->val_fmt || s.b_fmt != b->b_fmt)
                                     ? DASPMM_ERR_INVALID
                                     : batch_fill(s, &hi[i], wcap);
        if (fs != DASPMM_OK) {
            delete b;
            return fs;
        }
        const int w = hi[i].W;
        b->W = (i == 0 || b->W == w) ? w : 0;  // 0: widths differ
        b->grp = b->grp && hi[i].grp;
        b->total_nnz += s.nnz;
    }
    // Tiles from each rowPtr (copied to the host once).
    std::vector<BatchTile> tiles;
    std::vector<size_t> tile_off(n), slot_off(n), cnt_off(n);
    size_t nslot = 0, ncnt = 0;
    std::vector<long long> begin(n + 1, 0);
    {
        std::vector<int> rp;
        TilePlan plan;
        for (int i = 0; i < n; ++i) {
            const daspmm_instance &s = inst[i];
            rp.resize((size_t)s.nr + 1);
            if (s.nr > 0) {
                const cudaError_t e = cudaMemcpyAsync(rp.data(), s.rowPtr, sizeof(int) * (s.nr + 1),
                                                      cudaMemcpyDeviceToHost, st);
                const cudaError_t e2 = e == cudaSuccess ? cudaStreamSynchronize(st) : e;
                if (e2 != cudaSuccess) {
                    delete b;
                    return cuda_fail(e2);
                }
                if (rp[0] != 0 || rp[s.nr] != s.nnz) {
                    delete b;
                    return DASPMM_ERR_BAD_MATRIX;
                }
                for (int r = 0; r < s.nr; ++r)
                    if (rp[r + 1] < rp[r]) {
                        delete b;
                        return DASPMM_ERR_BAD_MATRIX;
                    }
            }
            build_tiles(rp.data(), s.nr, b->chunk, &plan);
            tile_off[i] = tiles.size();
            slot_off[i] = nslot;
            cnt_off[i] = ncnt;
            tiles.insert(tiles.end(), plan.tiles.begin(), plan.tiles.end());
            nslot += (size_t)plan.npieces * s.nv;
            ncnt += (size_t)plan.nlong * hi[i].col_tiles;
            hi[i].ntiles = (int)plan.tiles.size();
            begin[i + 1] = begin[i] + (long long)hi[i].ntiles * hi[i].col_tiles;
        }
    }
    b->nitems = begin[n];
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&b->d_head, sizeof(unsigned long long));
    if (e == cudaSuccess && n) e = cudaMalloc(&b->d_inst, sizeof(BatchInst) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_begin, sizeof(long long) * (n + 1));
    if (e == cudaSuccess && b->nitems) e = cudaMalloc(&b->d_items, sizeof(BatchItem) * b->nitems);
    if (e == cudaSuccess && !tiles.empty()) e = cudaMalloc(&b->d_tiles, sizeof(BatchTile) * tiles.size());
    if (e == cudaSuccess && nslot) e = cudaMalloc(&b->d_slots, sizeof(float) * nslot);
    if (e == cudaSuccess && ncnt) e = cudaMalloc(&b->d_cnt, sizeof(int) * ncnt);
    if (e != cudaSuccess) {
        cudaGetLastError();
        batch_free(b);
        return DASPMM_ERR_NOMEM;
    }
    for (int i = 0; i < n; ++i) {
        hi[i].tiles = b->d_tiles ? b->d_tiles + tile_off[i] : nullptr;
        hi[i].slots = b->d_slots ? b->d_slots + slot_off[i] : nullptr;
        hi[i].cnt = b->d_cnt ? b->d_cnt + cnt_off[i] : nullptr;
    }
    if (ncnt) e = cudaMemsetAsync(b->d_cnt, 0, sizeof(int) * ncnt, st);
    if (e == cudaSuccess && !tiles.empty())
        e = cudaMemcpyAsync(b->d_tiles, tiles.data(), sizeof(BatchTile) * tiles.size(),
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && n)
        e = cudaMemcpyAsync(b->d_inst, hi.data(), sizeof(BatchInst) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_begin, begin.data(), sizeof(long long) * (n + 1),
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const daspmm_status ps =
            batch_plan_async(b->d_inst, b->d_begin, n, b->d_items, b->nitems, st);
        if (ps != DASPMM_OK) {
            batch_free(b);
            return ps;
        }
        e = cudaStreamSynchronize(st);  // host vectors go out of scope
    }
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

}  // extern "C"

namespace daspmm {
// The fastest of `chunks` for these instances at the column-tile setting of
// `base` (lanes_col), each timed over `reps` runs after two warm-ups.
daspmm_status batch_tune_chunks(const daspmm_instance *inst, int n, const int *chunks,
                                int nchunks, daspmm_config base, int reps, int *best_chunk,
                                float *best_us, void *stream)
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
        daspmm_config cfg = base;
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
}  // namespace daspmm

extern "C" {

daspmm_status daspmm_batch_tune(const daspmm_instance *inst, int n, const int *chunks,
                                int nchunks, int reps, int *best_chunk, float *best_us,
                                void *stream)
{
    if (!best_chunk) return DASPMM_ERR_INVALID;
    return batch_tune_chunks(inst, n, chunks, nchunks, daspmm_config{}, reps, best_chunk,
                             best_us, stream);
}

daspmm_status daspmm_batch_tune_ex(const daspmm_instance *inst, int n, const int *chunks,
                                   int nchunks, const int *widths, int nwidths, int reps,
                                   daspmm_config *best, float *best_us, void *stream)
{
    static const int kChunks[] = {128, 256, 512, 1024};
    static const int kWidths[] = {128, 64, 32};
    if (!chunks || nchunks <= 0) {
        chunks = kChunks;
        nchunks = 4;
    }
    if (!widths || nwidths <= 0) {
        widths = kWidths;
        nwidths = 3;
    }
    if (!best || reps < 0) return DASPMM_ERR_INVALID;
    for (int w = 0; w < nwidths; ++w)
        if (widths[w] != 32 && widths[w] != 64 && widths[w] != 128) return DASPMM_ERR_INVALID;
    float bus = 0.0f;
    bool have = false;
    daspmm_config bc{};
    for (int w = 0; w < nwidths; ++w) {
        int ch = 0;
        float us = 0.0f;
        daspmm_config c{};
        c.lanes_col = widths[w] / 4;
        daspmm_status s = batch_tune_chunks(inst, n, chunks, nchunks, c, reps, &ch, &us, stream);
        if (s != DASPMM_OK) return s;
        if (!have || us < bus) {
            have = true;
            bus = us;
            bc = c;
            bc.chunk = ch;
        }
    }
    *best = bc;
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
