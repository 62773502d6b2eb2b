// gather_lean.cuh -- balanced-CSR SpMM, lean register gather at high occupancy.
//
// Measured on B200: gathering the B rows of the 262,144-row power-law matrix
// in its own column order runs at ~16 TB/s out of L2 when every SM keeps 64
// warps resident with 4 independent 16-byte loads per lane in flight; the
// bottleneck of a gather kernel is therefore warps in flight and instructions
// per nonzero, not the memory system.  This kernel keeps both small: one warp
// per chunk of the balanced split (k_partition), U = 4 nonzeros per step with
// their column/value loads broadcast to all lanes (one L1 line serves the
// warp), one W/32-float vector of the B row per lane, row ends from a
// 32-entry lane cache, and at most 48 registers per thread (40 warps per SM;
// measured better than 32 or 48 warps with fewer registers).
//
// Same chunk boundaries, walk and ownership as k_bal.  A row split across
// chunks is finished inside this kernel: its last piece to arrive adds all
// pieces in chunk order (piece_arrive), so no fix-up launch is needed.
// Row-major, nv % W == 0, B and C 16-byte aligned.
//
// Storage types (mixed precision): values TV in {float, bf16, fp16}, B in
// TB in {float, bf16, fp16, fp8 e4m3}; products and sums are FP32.  For FP8
// B, column k carries an FP32 scale (B = q * scale[k]); sums are taken over
// the unscaled q and each output column is scaled once, when its row is
// stored.  With KAHAN, rows of at least kahan_min nonzeros are summed with
// Kahan compensation (each piece of a split row included).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "internal.h"
#include "kernels.cuh"
#include "tma.cuh"

namespace daspmm {

using bf16 = __nv_bfloat16;
using fp16 = __half;
using fp8 = __nv_fp8_e4m3;

// 8 consecutive floats (32 bytes, 32-byte aligned).
__device__ __forceinline__ void ld8_nc(float (&r)[8], const float *p)
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]),
          "=f"(r[7])
        : "l"(p));
}
__device__ __forceinline__ void ld8_cg(float (&r)[8], const float *p)
{
    asm volatile("ld.global.cg.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]),
                   "=f"(r[6]), "=f"(r[7])
                 : "l"(p)
                 : "memory");
}
__device__ __forceinline__ void st8(float *p, const float (&r)[8])
{
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(r[0]),
                 "f"(r[1]), "f"(r[2]), "f"(r[3]), "f"(r[4]), "f"(r[5]), "f"(r[6]), "f"(r[7])
                 : "memory");
}
__device__ __forceinline__ void st8_hint(float *p, const float (&r)[8], uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8}, %9;" ::
                     "l"(p), "f"(r[0]), "f"(r[1]), "f"(r[2]), "f"(r[3]), "f"(r[4]), "f"(r[5]),
                 "f"(r[6]), "f"(r[7]), "l"(pol)
                 : "memory");
}

// N consecutive elements of B (storage type T) as floats, one vector load.
template <typename T, int N>
__device__ __forceinline__ void ld_b(float (&r)[N], const T *p)
{
    if constexpr (std::is_same<T, float>::value) {
        if constexpr (N == 8) ld8_nc(r, reinterpret_cast<const float *>(p));
        else ld_nc<N>(r, reinterpret_cast<const float *>(p));
    } else if constexpr (sizeof(T) == 2) {
        // 2-byte types: N = 8 -> 16 bytes, 4 -> 8 bytes, 2 -> 4 bytes, 1 -> 2 bytes
        uint32_t w[(N + 1) / 2];
        if constexpr (N == 8) {
            const uint4 t = __ldg(reinterpret_cast<const uint4 *>(p));
            w[0] = t.x; w[1] = t.y; w[2] = t.z; w[3] = t.w;
        } else if constexpr (N == 4) {
            const uint2 t = __ldg(reinterpret_cast<const uint2 *>(p));
            w[0] = t.x; w[1] = t.y;
        } else if constexpr (N == 2) {
            w[0] = __ldg(reinterpret_cast<const unsigned int *>(p));
        } else {
            w[0] = __ldg(reinterpret_cast<const unsigned short *>(p));
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const unsigned short h = (unsigned short)(w[i / 2] >> (16 * (i & 1)));
            if constexpr (std::is_same<T, bf16>::value) r[i] = __uint_as_float((uint32_t)h << 16);
            else r[i] = __half2float(__ushort_as_half(h));
        }
    } else {  // fp8 e4m3: N bytes
        uint32_t w[(N + 3) / 4];
        if constexpr (N == 8) {
            const uint2 t = __ldg(reinterpret_cast<const uint2 *>(p));
            w[0] = t.x; w[1] = t.y;
        } else if constexpr (N == 4) {
            w[0] = __ldg(reinterpret_cast<const unsigned int *>(p));
        } else if constexpr (N == 2) {
            w[0] = __ldg(reinterpret_cast<const unsigned short *>(p));
        } else {
            w[0] = __ldg(reinterpret_cast<const unsigned char *>(p));
        }
#pragma unroll
        for (int i = 0; i < N; i += 2) {
            const __half2_raw h2 = __nv_cvt_fp8x2_to_halfraw2(
                (__nv_fp8x2_storage_t)(w[i / 4] >> (8 * (i % 4))), __NV_E4M3);
            const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&h2));
            r[i] = f.x;
            if (i + 1 < N) r[i + 1] = f.y;
        }
    }
}

// (column tile, chunk) of a tile-major work item.
static __device__ __noinline__ int2 item_of(long long item, int nchunks)
{
    const int tile = (int)(item / nchunks);
    return make_int2(tile, (int)(item - (long long)tile * nchunks));
}

// One value of A (storage type T) as float, L2 hint.
template <typename T>
__device__ __forceinline__ float ld_val(const T *p, uint64_t pol)
{
    if constexpr (std::is_same<T, float>::value) {
        return ld_hint_f32(reinterpret_cast<const float *>(p), pol);
    } else {
        unsigned short h;
        asm("ld.global.nc.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(h) : "l"(p), "l"(pol));
        if constexpr (std::is_same<T, bf16>::value) return __uint_as_float((uint32_t)h << 16);
        else return __half2float(__ushort_as_half(h));
    }
}

#ifndef DASPMM_LEAN_MINB
#define DASPMM_LEAN_MINB 5  // CTAs of 256 threads per SM: 40 warps, <= 48 registers
#endif
#ifndef DASPMM_LEAN_U
#define DASPMM_LEAN_U 4     // nonzeros (B rows) in flight per warp step
#endif

// One chunk of the balanced split, column tile `tile` of `tiles`, summed by
// the whole warp with the per-nonzero walk: every nonzero is compared with
// the end of the current row (row ends from a 32-entry lane cache), so empty
// rows, beta != 0 and Kahan rows are all handled.  A row split across chunks
// leaves its pieces in carry slots; the last piece to arrive adds them all
// in chunk order (piece_arrive).  W / 32 elements of the B row per lane.
template <int W, int U, typename TV, typename TB, bool KAHAN>
__device__ __forceinline__ void lean_chunk(const KArgs &a, int c, int tile, int tiles,
                                           uint64_t pol_once)
{
    constexpr int VL = W / 32;  // elements of the B row per lane
    constexpr bool SCALED = std::is_same<TB, fp8>::value;
    const int lane = threadIdx.x & 31;
    const int tb = tile * W + lane * VL;
    const TB *Bl = reinterpret_cast<const TB *>(a.B) + tb;
    const TV *Av = reinterpret_cast<const TV *>(a.vals);
    float sc[VL];
#pragma unroll
    for (int e = 0; e < VL; ++e) sc[e] = SCALED ? __ldg(a.bscale + tb + e) : 1.0f;
    const int2 m0 = a.meta[c], m1 = a.meta[c + 1];
    const int k0 = m0.x, k1 = m1.x, s1 = m1.y;
    int r = m0.y;
    bool cont = k0 > __ldg(a.rowPtr + r);
    // row-end cache: lane l holds rowPtr[rb + 1 + l]; the next 32 are prefetched
    int rb = r;
    int rc = __ldg(a.rowPtr + min(rb + 1 + lane, a.nr));
    int rn = __ldg(a.rowPtr + min(rb + 33 + lane, a.nr));
    int re = __shfl_sync(kFull, rc, 0);
    float acc[VL], comp[VL];
#pragma unroll
    for (int e = 0; e < VL; ++e) acc[e] = comp[e] = 0.0f;
    // Kahan rows: length of the current row (its start is the previous end)
    int rs = KAHAN ? __ldg(a.rowPtr + r) : 0;
    bool kh = KAHAN && re - rs >= a.kahan_min;

    const bool head_piece = cont;  // row m0.y continues from an earlier chunk
    auto emit = [&](int row, bool ends) {
        if constexpr (SCALED) {
#pragma unroll
            for (int e = 0; e < VL; ++e) acc[e] *= sc[e];
        }
        if (ends && !cont) {
            float *dst = a.C + (size_t)row * a.ldc + tb;
            if (a.beta != 0.0f) {
                float old[VL];
                ld_plain<VL>(old, dst);
#pragma unroll
                for (int e = 0; e < VL; ++e) acc[e] = fmaf(a.beta, old[e], acc[e]);
            }
            st_hint<VL>(dst, acc, pol_once);
        } else {  // a piece of a row split across chunks: park it in its carry slot
            st_v<VL>(slot_ptr(a, c, cont ? 0 : 1, tb), acc);
        }
#pragma unroll
        for (int e = 0; e < VL; ++e) acc[e] = comp[e] = 0.0f;
        cont = false;
    };
    auto step = [&](int p, float v, const float (&b)[VL]) {
        while (p >= re) {
            emit(r, true);
            ++r;
            if (r - rb >= 32) {
                rb += 32;
                rc = rn;
                rn = __ldg(a.rowPtr + min(rb + 33 + lane, a.nr));
            }
            if constexpr (KAHAN) rs = re;
            re = __shfl_sync(kFull, rc, r - rb);
            if constexpr (KAHAN) kh = re - rs >= a.kahan_min;
        }
        if (KAHAN && kh) {
#pragma unroll
            for (int e = 0; e < VL; ++e) {  // Kahan: carry the rounding error along
                const float y = fmaf(v, b[e], -comp[e]);
                const float t = acc[e] + y;
                comp[e] = (t - acc[e]) - y;
                acc[e] = t;
            }
        } else {
#pragma unroll
            for (int e = 0; e < VL; ++e) acc[e] = fmaf(v, b[e], acc[e]);
        }
    };
    // Windows of 32 nonzeros: lane l holds the column/value of nonzero
    // wb + l; the next window's are loaded while this one is gathered.
    auto load_win = [&](int wb, int &col, float &val) {
        const bool ok = wb + lane < k1;
        col = ok ? ld_hint_s32(a.colIdx + wb + lane, pol_once) : 0;
        val = ok ? ld_val<TV>(Av + wb + lane, pol_once) : 0.0f;
    };
    int ccur, cnext;
    float vcur, vnext;
    load_win(k0, ccur, vcur);
    for (int wb = k0; wb < k1; wb += 32) {
        load_win(wb + 32, cnext, vnext);
        const int cnt = min(32, k1 - wb);
        int t = 0;
        for (; t + U <= cnt; t += U) {  // U rows in flight
            int cc[U];
            float vv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                cc[u] = __shfl_sync(kFull, ccur, t + u);
                vv[u] = __shfl_sync(kFull, vcur, t + u);
            }
            float b[U][VL];
#pragma unroll
            for (int u = 0; u < U; ++u) ld_b<TB, VL>(b[u], Bl + (size_t)cc[u] * a.ldb);
#pragma unroll
            for (int u = 0; u < U; ++u) step(wb + t + u, vv[u], b[u]);
        }
        for (; t < cnt; ++t) {
            float b[VL];
            ld_b<TB, VL>(b, Bl + (size_t)__shfl_sync(kFull, ccur, t) * a.ldb);
            step(wb + t, __shfl_sync(kFull, vcur, t), b);
        }
        ccur = cnext;
        vcur = vnext;
    }
    while (r < s1) {
        emit(r, true);
        ++r;
    }
    const int head_row = m0.y;
    bool tail_piece = false;
    if (r < a.nr && r == s1 && __ldg(a.rowPtr + r) < k1) {
        tail_piece = !cont;  // a continuing row here is the head piece itself
        emit(r, false);
    }
    // the pieces this chunk parked arrive (at most two; fence + count, and
    // the last piece of a row adds them all)
    if (head_piece) piece_arrive<VL>(a, head_row, tb, tiles, tile);
    if (tail_piece) piece_arrive<VL>(a, s1, tb, tiles, tile);
}

template <int W, int U, typename TV = float, typename TB = float, bool KAHAN = false>
__global__ void __launch_bounds__(256, DASPMM_LEAN_MINB) k_bal_lean(const KArgs a)
{
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const uint64_t pol_once = policy_evict_first();
    pdl_wait();  // the boundaries (k_partition) or the list (k_bal_fast) are complete
    // Queue mode: chunks are handed out dynamically -- each warp starts with
    // chunk = its index, then takes the next unclaimed one from the column
    // tile's queue head (zeroed by k_partition), so warps that draw short
    // chunks take more and no wave of chunks is left half-used.  List mode:
    // the chunks k_bal_fast left over (a.list), strided over the warps.
    // Plan mode (2): the list is the planned product's fixed list of chunks
    // with an empty row, unless row 0 of B holds an Inf or NaN -- then the
    // window kernel took no chunk and every chunk is walked here.
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    bool all = false;
    if (a.list_mode == 2) {
        bool pad_ok = true;
        for (int k = lane; a.nnz > 0 && k < a.nv; k += 32) {
            float x[1];
            ld_b<TB, 1>(x, reinterpret_cast<const TB *>(a.B) + k);
            pad_ok &= isfinite(x[0]);
        }
        all = !__all_sync(kFull, pad_ok);
    }
    const long long limit = (a.list_mode && !all) ? (long long)a.list[0] : (long long)a.nchunks;
    long long cl = wid;
    while (cl < limit) {
        const int c = (a.list_mode && !all) ? a.list[1 + cl] : (int)cl;
        lean_chunk<W, U, TV, TB, KAHAN>(a, c, blockIdx.y, gridDim.y, pol_once);
        if (a.list_mode) {
            cl += nwarps;  // listed chunks (or, plan mode with a non-finite row 0, all)
        } else {
            unsigned int nx = 0;
            if (lane == 0) nx = atomicAdd(a.head + blockIdx.y, 1u);
            cl = nwarps + (long long)__shfl_sync(kFull, nx, 0);
        }
    }
}

// Balanced-CSR SpMM, beta == 0, for chunks without empty rows: the ends of
// the rows finishing in a window of 32 nonzeros come as one bitmask (lane l
// looks at the end of row r + l; with no empty row the 32 lanes cover every
// row that can end in the window), so the window is summed straight through
// -- no per-nonzero test against a row end -- and a row is stored at its bit.
// A chunk holding an empty row is left untouched and listed in a.list for
// k_bal_lean (list mode), launched after this kernel.  Same chunks, carries
// and split-row combine as k_bal_lean, so results are identical to it.
template <int W, int U, typename TV = float, typename TB = float>
__global__ void __launch_bounds__(256, DASPMM_LEAN_MINB) k_bal_fast(const KArgs a)
{
    constexpr int VL = W / 32;
    constexpr bool SCALED = std::is_same<TB, fp8>::value;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const TV *Av = reinterpret_cast<const TV *>(a.vals);
    const uint64_t pol_once = policy_evict_first();
    // Column tiles: W = 128 takes its tile from blockIdx.y (the CTAs of tile 0
    // are scheduled first, so the tiles are gathered roughly one after the
    // other).  Narrower tiles run one queue of (tile, chunk) items, tile-major,
    // decoded out of line: measured 25-35 % faster for W = 64 and 32 (N = 32,
    // 64, 192 on the power-law matrix), slower for W = 128.
    const int tiles = W == 128 ? (int)gridDim.y : a.nv / W;
    const long long limit = W == 128 ? (long long)a.nchunks : (long long)a.nchunks * tiles;

    pdl_trigger();  // the list-mode walk may be scheduled; it waits for this grid
    pdl_wait();     // the boundaries from k_partition are complete
    // A chunk's last window is padded with column 0, value 0: that adds
    // nothing unless row 0 of B holds an Inf or NaN (0 * Inf = NaN).  Then
    // every chunk is handed to the walk kernel, which never pads (the same
    // decision in every warp and column tile).  Without nonzeros nothing is
    // padded (and B may have no rows).
    bool pad_ok = true;
    for (int k = lane; a.nnz > 0 && k < a.nv; k += 32) {
        float x[1];
        ld_b<TB, 1>(x, reinterpret_cast<const TB *>(a.B) + k);
        pad_ok &= isfinite(x[0]);
    }
    pad_ok = __all_sync(kFull, pad_ok);
    long long cl = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    while (cl < limit) {
        int tile, c;
        if constexpr (W == 128) {
            tile = blockIdx.y;
            c = (int)cl;
        } else {
            const int2 tc = item_of(cl, a.nchunks);
            tile = tc.x;
            c = tc.y;
        }
        const int tb = tile * W + lane * VL;
        const TB *Bl = reinterpret_cast<const TB *>(a.B) + tb;
        float sc[VL];
#pragma unroll
        for (int e = 0; e < VL; ++e) sc[e] = SCALED ? __ldg(a.bscale + tb + e) : 1.0f;
        const int2 m0 = a.meta[c], m1 = a.meta[c + 1];
        const int k0 = m0.x, k1 = m1.x, s1 = m1.y;
        int r = m0.y;
        const int rstart = __ldg(a.rowPtr + r);
        // ends of rows r .. r+31; any empty row among [r, s1) hands the chunk on
        int E = __ldg(a.rowPtr + min(r + 1 + lane, a.nr));
        bool empty_row;
        {
            int prev = __shfl_up_sync(kFull, E, 1);
            if (lane == 0) prev = rstart;
            empty_row = __any_sync(kFull, r + lane < s1 && E == prev);
            int last = __shfl_sync(kFull, E, 31);
            for (int rb = r + 32; !empty_row && rb < s1; rb += 32) {
                const int e2 = __ldg(a.rowPtr + min(rb + 1 + lane, a.nr));
                int p2 = __shfl_up_sync(kFull, e2, 1);
                if (lane == 0) p2 = last;
                empty_row = __any_sync(kFull, rb + lane < s1 && e2 == p2);
                last = __shfl_sync(kFull, e2, 31);
            }
        }
        if (empty_row || !pad_ok) {
            if (tile == 0 && lane == 0) a.list[1 + atomicAdd(a.list, 1)] = c;  // every tile
        } else {
            bool cont = k0 > rstart;
            const bool head_piece = cont;
            float acc[VL];
#pragma unroll
            for (int e = 0; e < VL; ++e) acc[e] = 0.0f;
            auto load_win = [&](int wb, int &col, float &val) {
                const bool ok = wb + lane < k1;
                col = ok ? ld_hint_s32(a.colIdx + wb + lane, pol_once) : 0;
                val = ok ? ld_val<TV>(Av + wb + lane, pol_once) : 0.0f;
            };
            int ccur, cnext;
            float vcur, vnext;
            load_win(k0, ccur, vcur);
            for (int wb = k0; wb < k1; wb += 32) {
                load_win(wb + 32, cnext, vnext);
                const int cnt = min(32, k1 - wb);
                const int pos = E - 1 - wb;
                const bool in = r + 1 + lane <= a.nr && pos >= 0 && pos < cnt;
                const unsigned ends = __reduce_or_sync(kFull, in ? (1u << pos) : 0u);
                // the next window's row ends load while this one is summed
                E = __ldg(a.rowPtr + min(r + __popc(ends) + 1 + lane, a.nr));
                float *cdst = cont ? slot_ptr(a, c, 0, tb) : a.C + (size_t)r * a.ldc + tb;
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
                    for (int u = 0; u < U; ++u) ld_b<TB, VL>(b[u], Bl + (size_t)cc[u] * a.ldb);
#pragma unroll
                    for (int u = 0; u < U; ++u) {
#pragma unroll
                        for (int e = 0; e < VL; ++e) acc[e] = fmaf(vv[u], b[u][e], acc[e]);
                        if ((ends >> (g * U + u)) & 1u) {
                            if constexpr (SCALED) {
#pragma unroll
                                for (int e = 0; e < VL; ++e) acc[e] *= sc[e];
                            }
                            st_hint<VL>(cdst, acc, pol_once);
#pragma unroll
                            for (int e = 0; e < VL; ++e) acc[e] = 0.0f;
                            cont = false;
                            ++r;
                            cdst = a.C + (size_t)r * a.ldc + tb;
                        }
                    }
                    // keep the next group's loads behind this group (registers)
                    asm volatile("" ::: "memory");
                }
                ccur = cnext;
                vcur = vnext;
            }
            // every row of [m0.y, s1) has been stored; row s1 may continue
            bool tail_piece = false;
            if (r < a.nr && r == s1 && __ldg(a.rowPtr + r) < k1) {
                if constexpr (SCALED) {
#pragma unroll
                    for (int e = 0; e < VL; ++e) acc[e] *= sc[e];
                }
                tail_piece = !cont;  // a continuing row here is the head piece itself
                st_v<VL>(slot_ptr(a, c, cont ? 0 : 1, tb), acc);
            }
            if (head_piece)
                piece_arrive_ool<VL>(a.rowPtr, a.cnt, a.slots, a.C, a.ldc, a.nv, a.chunk, 0.0f,
                                     m0.y, tb, tiles, tile);
            if (tail_piece)
                piece_arrive_ool<VL>(a.rowPtr, a.cnt, a.slots, a.C, a.ldc, a.nv, a.chunk, 0.0f,
                                     s1, tb, tiles, tile);
        }
        unsigned int nx = 0;
        if (lane == 0) nx = atomicAdd(a.head + (W == 128 ? blockIdx.y : 0), 1u);
        cl = nwarps + (long long)__shfl_sync(kFull, nx, 0);
    }
}

// ---------------------------------------------------------------- half-warp form
// VL floats: plain / L2-hinted stores and L2-coherent loads, VL <= 8.
// (VL = 16: two 32-byte accesses)
template <int VL>
__device__ __forceinline__ void st_n(float *p, const float (&r)[VL])
{
    if constexpr (VL == 16) {
        st8(p, *reinterpret_cast<const float(*)[8]>(&r[0]));
        st8(p + 8, *reinterpret_cast<const float(*)[8]>(&r[8]));
    } else if constexpr (VL == 8) {
        st8(p, r);
    } else {
        st_v<VL>(p, r);
    }
}
template <int VL>
__device__ __forceinline__ void st_hint_n(float *p, const float (&r)[VL], uint64_t pol)
{
    if constexpr (VL == 16) {
        st8_hint(p, *reinterpret_cast<const float(*)[8]>(&r[0]), pol);
        st8_hint(p + 8, *reinterpret_cast<const float(*)[8]>(&r[8]), pol);
    } else if constexpr (VL == 8) {
        st8_hint(p, r, pol);
    } else {
        st_hint<VL>(p, r, pol);
    }
}
template <int VL>
__device__ __forceinline__ void ld_cg_n(float (&r)[VL], const float *p)
{
    if constexpr (VL == 16) {
        ld8_cg(*reinterpret_cast<float(*)[8]>(&r[0]), p);
        ld8_cg(*reinterpret_cast<float(*)[8]>(&r[8]), p + 8);
    } else if constexpr (VL == 8) {
        ld8_cg(r, p);
    } else {
        ld_cg<VL>(r, p);
    }
}

// NW 32-bit words (NW = 8: one 32-byte load, 4: 16 bytes, 2: 8 bytes) of B,
// read-only path, left packed; elem<TB>() unpacks element i as a float.
template <int NW>
__device__ __forceinline__ void ld_raw(uint32_t (&w)[NW], const void *p)
{
    if constexpr (NW == 8) {
        float f[8];
        ld8_nc(f, reinterpret_cast<const float *>(p));
#pragma unroll
        for (int i = 0; i < 8; ++i) w[i] = __float_as_uint(f[i]);
    } else if constexpr (NW == 4) {
        const uint4 t = __ldg(reinterpret_cast<const uint4 *>(p));
        w[0] = t.x; w[1] = t.y; w[2] = t.z; w[3] = t.w;
    } else if constexpr (NW == 2) {
        const uint2 t = __ldg(reinterpret_cast<const uint2 *>(p));
        w[0] = t.x; w[1] = t.y;
    } else {
        static_assert(NW == 1, "4-, 8-, 16- or 32-byte lane loads");
        w[0] = __ldg(reinterpret_cast<const unsigned int *>(p));
    }
}
// acc[0] += a * lo(w), acc[1] += a * hi(w) for two packed 16-bit B elements
// and a 16-bit value a of the same type (BF16 or FP16), FP32 accumulate in one
// instruction each (fma.rn.f32.bf16 / .f16, sm_100): the product of two 16-bit
// values is exact in FP32, so each result is the single rounding of
// a*b + acc -- bit-identical to fmaf on the widened operands.
template <typename T>
__device__ __forceinline__ void fma2_16(float &acc0, float &acc1, unsigned short a, uint32_t w)
{
    unsigned short lo, hi;
    asm("mov.b32 {%0, %1}, %2;" : "=h"(lo), "=h"(hi) : "r"(w));
    if constexpr (std::is_same<T, bf16>::value) {
        asm("fma.rn.f32.bf16 %0, %1, %2, %0;" : "+f"(acc0) : "h"(a), "h"(lo));
        asm("fma.rn.f32.bf16 %0, %1, %2, %0;" : "+f"(acc1) : "h"(a), "h"(hi));
    } else {
        asm("fma.rn.f32.f16 %0, %1, %2, %0;" : "+f"(acc0) : "h"(a), "h"(lo));
        asm("fma.rn.f32.f16 %0, %1, %2, %0;" : "+f"(acc1) : "h"(a), "h"(hi));
    }
}

template <typename TB, int NW>
__device__ __forceinline__ float elem(const uint32_t (&w)[NW], int i)
{
    if constexpr (std::is_same<TB, float>::value) {
        return __uint_as_float(w[i]);
    } else if constexpr (std::is_same<TB, bf16>::value) {
        const uint32_t x = w[i >> 1];
        return __uint_as_float((i & 1) ? (x & 0xFFFF0000u) : (x << 16));
    } else if constexpr (std::is_same<TB, fp16>::value) {
        return __half2float(__ushort_as_half((unsigned short)(w[i >> 1] >> (16 * (i & 1)))));
    } else {  // fp8 e4m3 (element pairs share one conversion; see elem2)
        const __half2_raw h2 = __nv_cvt_fp8x2_to_halfraw2(
            (__nv_fp8x2_storage_t)(w[i >> 2] >> (8 * (i & 2))), __NV_E4M3);
        const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&h2));
        return (i & 1) ? f.y : f.x;
    }
}

// piece_arrive for a G-lane worker of a warp (lanes of `gmask`, VL floats per
// lane at column `col`), beta == 0: the same counters, carries and order of
// summation as piece_arrive, so the two combine pieces of one row freely.
// Templated on the kernel's types so that every kernel has its own copy:
// ptxas 12.9 crashes (at build time) on one copy shared by two kernels.
template <int G, int VL, typename TV, typename TB>
static __device__ __noinline__ void piece_arrive_grp(const int *__restrict__ rowPtr, int *cnt,
                                                     const float *slots, float *C, int ldc,
                                                     int nv, int chunk, int row, int col,
                                                     int tiles, int tile, unsigned gmask)
{
    const int rs = __ldg(rowPtr + row), re = __ldg(rowPtr + row + 1);
    const int c0 = first_chunk(rs, chunk), c1 = last_chunk(re, chunk);
    __threadfence();
    __syncwarp(gmask);
    int last = 0;
    if ((threadIdx.x & (G - 1)) == 0) last = atomicAdd(cnt + (size_t)c0 * tiles + tile, 1) == c1 - c0;
    last = __shfl_sync(gmask, last, 0, G);
    if (!last) return;
    // every piece has arrived: the counter goes back to zero for the next call
    if ((threadIdx.x & (G - 1)) == 0) cnt[(size_t)c0 * tiles + tile] = 0;
    __threadfence();
    float tot[VL];
    ld_cg_n<VL>(tot, slots + ((size_t)c0 * 2 + 1) * nv + col);
    constexpr int P = 2;  // independent carry loads in flight
    for (int cb = c0 + 1; cb <= c1; cb += P) {
        float hp[P][VL];
#pragma unroll
        for (int u = 0; u < P; ++u)
            if (cb + u <= c1) ld_cg_n<VL>(hp[u], slots + ((size_t)(cb + u) * 2) * nv + col);
#pragma unroll
        for (int u = 0; u < P; ++u)
            if (cb + u <= c1)
#pragma unroll
                for (int e = 0; e < VL; ++e) tot[e] += hp[u][e];
    }
    st_n<VL>(C + (size_t)row * ldc + col, tot);
}

#ifndef DASPMM_GRP
#define DASPMM_GRP 1        // FP32 32/64/128-column tiles take the worker-group kernel
#endif
#ifndef DASPMM_GRP_U
#define DASPMM_GRP_U 8      // nonzeros in flight per worker step
#endif
#ifndef DASPMM_GRP_U16
#define DASPMM_GRP_U16 16   // 2-byte B (8 elements per 16-byte lane load)
#endif
#ifndef DASPMM_GRP_U8
#define DASPMM_GRP_U8 8     // 1-byte B (16 elements per 16-byte lane load)
#endif
#ifndef DASPMM_GRP_MINB
#define DASPMM_GRP_MINB 2   // CTAs of 256 threads per SM: 16 warps, <= 128 registers
#endif

// k_bal_fast with G-lane workers, beta == 0.  Each worker (G consecutive
// lanes) takes one chunk of a group (32/G consecutive chunks per warp) and
// covers its column tile of a B row with G lanes x one 16- or 32-byte load
// of EPL elements each (FP32: 8 per 32 bytes; BF16 / FP16: 16 per 32 bytes;
// E4M3: 16 per 16 bytes), so the tile is G*EPL columns and one warp
// instruction gathers 32/G nonzeros.  FP32 uses G = 16 for 128-column tiles
// and G = 8 for 64; BF16 / FP16 / E4M3 reach 128 columns with G = 8.  The
// workers run in step: the window loop runs to the longest chunk of the group
// (balanced chunks differ by a few nonzeros); a worker past its chunk's end
// gathers padding (column 0, value 0) and stores nothing.  Windows are G
// nonzeros (lane l of a worker ends row r + l), gathered min(U, G) B rows at a
// time, each row's EPL elements unpacked to FP32 as they are summed.
// Everything else is k_bal_fast's: same chunks, carries, split-row combine
// and order of summation (FP32 products and sums), so results are
// bit-identical to it.  Column tiles are blockIdx.y: the CTAs of tile 0 are
// dispatched first, so with several tiles their B column slabs are gathered
// one after the other.  B aligned to EPL*sizeof(TB) bytes, C and the carry
// slots to 32 bytes.
template <int G, int EPL, int U, typename TV = float, typename TB = float,
          int MINB = DASPMM_GRP_MINB, bool WS = false>
__global__ void __launch_bounds__(256, MINB) k_bal_grp(const KArgs a)
{
    constexpr int NW = 32 / G;                             // workers per warp
    constexpr int RAW = EPL * (int)sizeof(TB) / 4;         // 32-bit words per lane load
    constexpr int UU = U < G ? U : G;                      // rows in flight per step
    constexpr unsigned GM = G == 32 ? 0xFFFFFFFFu : ((1u << G) - 1u);
    constexpr bool SCALED = std::is_same<TB, fp8>::value;
    // FP16 values and B: one mixed-precision FMA per element (measured 2-3%
    // faster at N = 256 / 512; the BF16 form of that instruction measured
    // slower than unpacking to FP32, so BF16 unpacks)
    constexpr bool PAIR16 = std::is_same<TV, fp16>::value && std::is_same<TB, fp16>::value;
    const int lane = threadIdx.x & 31, w = lane / G, gl = lane % G;
    const unsigned gmask = GM << (G * w);
    const int tile = blockIdx.y, tiles = gridDim.y;
    const int tb = tile * (G * EPL) + gl * EPL;
    const TB *Bl = reinterpret_cast<const TB *>(a.B) + tb;
    const TV *Av = reinterpret_cast<const TV *>(a.vals);
    const uint64_t pol_once = policy_evict_first();
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long ngroups = ((long long)a.nchunks + NW - 1) / NW;

    pdl_trigger();  // the list-mode walk may be scheduled; it waits for this grid
    pdl_wait();     // the boundaries from k_partition are complete
    float sc[SCALED ? EPL : 1];  // read after the wait, like every input
#pragma unroll
    for (int e = 0; e < (SCALED ? EPL : 1); ++e) sc[e] = SCALED ? __ldg(a.bscale + tb + e) : 1.0f;
    // padding (column 0, value 0) adds nothing unless row 0 of B holds an Inf
    // or NaN; then every chunk is handed to the walk kernel (as in k_bal_fast).
    // Without nonzeros nothing is padded (and B may have no rows).
    bool pad_ok = true;
    for (int k = lane; a.nnz > 0 && k < a.nv; k += 32) {
        float x[1];
        ld_b<TB, 1>(x, reinterpret_cast<const TB *>(a.B) + k);
        pad_ok &= isfinite(x[0]);
    }
    pad_ok = __all_sync(kFull, pad_ok);
    long long gi = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    while (gi < ngroups) {
        const int c = (int)(NW * gi) + w;
        const bool have = c < a.nchunks;
        int k0 = 0, k1 = 0, s1 = 0, r = 0, rstart = 0;
        if (have) {
            const int2 m0 = a.meta[c], m1 = a.meta[c + 1];
            k0 = m0.x;
            k1 = m1.x;
            s1 = m1.y;
            r = m0.y;
            rstart = __ldg(a.rowPtr + r);
        }
        const int r0 = r;
        // ends of rows r .. r+G-1; any empty row among [r, s1) hands the chunk on
        int E = __ldg(a.rowPtr + min(r + 1 + gl, a.nr));
        bool empty_row;
        {
            int prev = __shfl_up_sync(kFull, E, 1, G);
            if (gl == 0) prev = rstart;
            empty_row = (__ballot_sync(kFull, have && r + gl < s1 && E == prev) & gmask) != 0;
            bool more = have && !empty_row && r + G < s1;
            if constexpr (WS) {
                // the rest of the chunk's rows, 32 per step: lane gl of a worker
                // checks rows rb + gl*K .. rb + gl*K + K - 1 (K + 1 independent
                // loads) -- one load latency per 32 rows instead of per G
                constexpr int K = 32 / G;
                for (int rb = r + G; __any_sync(kFull, more); rb += 32) {
                    bool e = false;
                    if (more) {
                        const int k0 = rb + gl * K;
                        int q[K + 1];
#pragma unroll
                        for (int j = 0; j <= K; ++j) q[j] = __ldg(a.rowPtr + min(k0 + j, a.nr));
#pragma unroll
                        for (int j = 0; j < K; ++j) e |= k0 + j < s1 && q[j + 1] == q[j];
                    }
                    const unsigned b2 = __ballot_sync(kFull, e);
                    if (more) empty_row = (b2 & gmask) != 0;
                    more = more && !empty_row && rb + 32 < s1;
                }
            } else {
                int last = __shfl_sync(kFull, E, G - 1, G);
                for (int rb = r + G; __any_sync(kFull, more); rb += G) {
                    int e2 = 0;
                    if (more) e2 = __ldg(a.rowPtr + min(rb + 1 + gl, a.nr));
                    int p2 = __shfl_up_sync(kFull, e2, 1, G);
                    if (gl == 0) p2 = last;
                    const unsigned b2 = __ballot_sync(kFull, more && rb + gl < s1 && e2 == p2);
                    if (more) empty_row = (b2 & gmask) != 0;
                    last = __shfl_sync(kFull, e2, G - 1, G);
                    more = more && !empty_row && rb + G < s1;
                }
            }
        }
        const bool skip = !have || empty_row || !pad_ok;
        // the walk kernel sums these; a planned product's list is fixed
        if (have && (empty_row || !pad_ok) && tile == 0 && gl == 0 && a.list_mode != 2)
            a.list[1 + atomicAdd(a.list, 1)] = c;  // every tile
        const int kb = skip ? 0 : k0, ke = skip ? 0 : k1;
        int nwin = (ke - kb + G - 1) / G;
#pragma unroll
        for (int o = G; o < 32; o <<= 1) nwin = max(nwin, __shfl_xor_sync(kFull, nwin, o));
        bool cont = !skip && k0 > rstart;
        const bool head_piece = cont;
        float acc[EPL];
#pragma unroll
        for (int e = 0; e < EPL; ++e) acc[e] = 0.0f;
        auto load_win = [&](int wb, int &col, float &val) {
            const bool ok = wb + gl < ke;
            col = ok ? ld_hint_s32(a.colIdx + wb + gl, pol_once) : 0;
            val = ok ? ld_val<TV>(Av + wb + gl, pol_once) : 0.0f;
        };
        int ccur, cnext;
        float vcur, vnext;
        int wb = kb;
        load_win(wb, ccur, vcur);
        for (int wi = 0; wi < nwin; ++wi, wb += G) {
            load_win(wb + G, cnext, vnext);
            const int cnt = ke - wb;  // nonzeros of this worker left (<= 0: idle)
            const int pos = E - 1 - wb;
            const bool in = r + 1 + gl <= a.nr && pos >= 0 && pos < min(cnt, G);
            const unsigned e32 = __reduce_or_sync(kFull, in ? (1u << (pos + G * w)) : 0u);
            const unsigned ends = (e32 >> (G * w)) & GM;
            // the next window's row ends load while this one is summed
            E = __ldg(a.rowPtr + min(r + __popc(ends) + 1 + gl, a.nr));
            float *cdst = cont ? slot_ptr(a, c, 0, tb) : a.C + (size_t)r * a.ldc + tb;
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
                for (int u = 0; u < UU; ++u) ld_raw<RAW>(b[u], Bl + (size_t)cc[u] * a.ldb);
#pragma unroll
                for (int u = 0; u < UU; ++u) {
                    if constexpr (PAIR16) {
                        // vv holds the FP16 value widened exactly: narrowing is exact
                        const unsigned short a16 = __half_as_ushort(__float2half_rn(vv[u]));
#pragma unroll
                        for (int i = 0; i < RAW; ++i)
                            fma2_16<TB>(acc[2 * i], acc[2 * i + 1], a16, b[u][i]);
                    } else {
#pragma unroll
                        for (int e = 0; e < EPL; ++e)
                            acc[e] = fmaf(vv[u], elem<TB, RAW>(b[u], e), acc[e]);
                    }
                    if ((ends >> (g * UU + u)) & 1u) {
                        if constexpr (SCALED) {
#pragma unroll
                            for (int e = 0; e < EPL; ++e) acc[e] *= sc[e];
                        }
                        st_hint_n<EPL>(cdst, acc, pol_once);
#pragma unroll
                        for (int e = 0; e < EPL; ++e) acc[e] = 0.0f;
                        cont = false;
                        ++r;
                        cdst = a.C + (size_t)r * a.ldc + tb;
                    }
                }
                asm volatile("" ::: "memory");
            }
            ccur = cnext;
            vcur = vnext;
        }
        // every row of [m0.y, s1) has been stored; row s1 may continue
        bool tail_piece = false;
        if (!skip && r < a.nr && r == s1 && __ldg(a.rowPtr + r) < k1) {
            tail_piece = !cont;  // a continuing row here is the head piece itself
            if constexpr (SCALED) {
#pragma unroll
                for (int e = 0; e < EPL; ++e) acc[e] *= sc[e];
            }
            st_n<EPL>(slot_ptr(a, c, cont ? 0 : 1, tb), acc);
        }
        if (head_piece)
            piece_arrive_grp<G, EPL, TV, TB>(a.rowPtr, a.cnt, a.slots, a.C, a.ldc, a.nv, a.chunk,
                                             r0, tb, tiles, tile, gmask);
        if (tail_piece)
            piece_arrive_grp<G, EPL, TV, TB>(a.rowPtr, a.cnt, a.slots, a.C, a.ldc, a.nv, a.chunk,
                                             s1, tb, tiles, tile, gmask);
        __syncwarp();
        // the next group from the tile's queue; a call makes exactly ngroups
        // claims, so a planned product counts on from where the last one ended
        unsigned int nx = 0;
        if (lane == 0) nx = atomicAdd(a.head + tile, 1u) - a.head_base;
        gi = nwarps + (long long)__shfl_sync(kFull, nx, 0);
    }
}

// A launch that may overlap the previous kernel of the stream (programmatic
// dependent launch); the kernel calls pdl_wait() before reading its inputs.
// With a.l2_window > 0 the launch also carries an L2 access-policy window
// over B (that many thousandths of its lines persisting, the rest streaming).
// A failure is left in the runtime's last error for the caller's check.
inline void launch_pdl(void (*kernel)(KArgs), dim3 grid, cudaStream_t st, const KArgs &a)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.numAttrs = 1;
    if (a.l2_window > 0 && a.b_bytes > 0) {
        int dev = 0, maxw = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, dev);
        at[1].id = cudaLaunchAttributeAccessPolicyWindow;
        at[1].val.accessPolicyWindow.base_ptr = const_cast<float *>(a.B);
        at[1].val.accessPolicyWindow.num_bytes = std::min<size_t>(a.b_bytes, (size_t)maxw);
        at[1].val.accessPolicyWindow.hitRatio = std::min(1.0f, a.l2_window / 1000.0f);
        at[1].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        at[1].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        cfg.numAttrs = maxw > 0 ? 2 : 1;
    }
    cfg.attrs = at;
    cudaLaunchKernelEx(&cfg, kernel, a);
}

// The worker-group kernel, when it takes this product: beta == 0, EPL
// elements of B per lane load (FP32: 8 in 32 bytes; BF16 / FP16: 8 in 16
// bytes; E4M3: 16 in 16 bytes), G = W / EPL lanes per chunk, U rows in
// flight per worker, stores of C and carries 32-byte aligned.  Returns false
// (nothing launched) otherwise.  Measured on the 262k power-law matrix: the
// group form wins for FP32 storage and 128- or 64-column tiles (N = 128: 84
// against 113 us, N = 64: 54 against 61 us); 32-column FP32 tiles take 8-lane
// workers with 16-byte loads at 24 warps per SM and the chunk scan 32 rows per
// step (N = 32: 34.3 against 41 us for the 32-lane kernel; 4-lane workers with
// 32-byte loads 42 us; on the 1M uniform-random matrix 187 against 293 us).
// 2-byte B: 16-lane workers with 16 rows in flight (the registers of 8 FP32
// rows hold 16 BF16 rows): BF16 N = 128 70.6 against 77.4 us (32-lane), FP16
// 62.5 against 76.4; N = 512 BF16 254 against 335, FP16 221 against 332.
// E4M3 B: for one 128-column tile 16-lane workers with 8-byte loads and 16
// rows in flight (N = 128: 64.6 against 69.8 us), for more tiles 8-lane
// workers with 16-byte loads (N = 512: 239 against 318 us; the 16-lane form
// 247).
template <int G, int EPL, int U, typename TV, typename TB, int MINB = DASPMM_GRP_MINB,
          bool WS = false>
inline bool launch_grp_as(const Resolved &r, const KArgs &a, cudaStream_t st)
{
    const bool aligned_g =
        (reinterpret_cast<uintptr_t>(a.B) % (EPL * sizeof(TB))) == 0 &&
        ((reinterpret_cast<uintptr_t>(a.C) | reinterpret_cast<uintptr_t>(a.slots)) % 32) == 0 &&
        a.ldb % EPL == 0 && a.ldc % 8 == 0 && a.nv % (G * EPL) == 0;
    if (!(DASPMM_GRP && a.beta == 0.0f && aligned_g)) return false;
    constexpr int NWK = 32 / G;
    const long long groups = ((long long)a.nchunks + NWK - 1) / NWK;
    const unsigned gg = (unsigned)std::max<long long>(
        1, std::min<long long>((groups + 7) / 8,
                               (long long)device_sms() * MINB));
    launch_pdl(k_bal_grp<G, EPL, U, TV, TB, MINB, WS>, dim3(gg, r.tiles), st, a);
    return true;
}

// Reduced-precision B in 32- and 64-column tiles: workers of W / E lanes with
// 8-byte lane loads of E elements (BF16 / FP16: 4, E4M3: 8), 3 CTAs per SM
// (24 warps, <= 85 registers).  Measured on the 262k power-law and the 1M
// uniform-random matrix against the 32-lane kernel (us): N = 32 BF16 35.1 /
// 152 against 47.0 / 278, FP16 34.8 / 150 against 47.1 / 278, E4M3 44.9 / 130
// against 48.4 / 228; N = 64 BF16 44.9 / 229 against 64.9 / 515, FP16 42.9 /
// 225 against 48.4 / 352, E4M3 45.6 / 197 against 49.9 / 304.  16-byte loads,
// 4-byte loads, and 2 or 4 CTAs per SM measured slower overall.  The chunk
// scan 32 rows per step pays except for FP16 (fma.rn.f32.f16) 32-column tiles.
template <int W, typename TV, typename TB>
inline bool launch_grp_narrow(const Resolved &r, const KArgs &a, cudaStream_t st)
{
    constexpr int E = sizeof(TB) == 2 ? 4 : 8;
    constexpr bool ws = !(W == 32 && std::is_same<TV, fp16>::value && std::is_same<TB, fp16>::value);
    return launch_grp_as<W / E, E, 16, TV, TB, 3, ws>(r, a, st);
}

template <int W, typename TV, typename TB>
inline bool launch_grp(const Resolved &r, const KArgs &a, cudaStream_t st)
{
    constexpr bool f32 = std::is_same<TV, float>::value && std::is_same<TB, float>::value;
    constexpr bool b16 = sizeof(TB) == 2;
    if constexpr (f32) {
        if constexpr (W >= 64) return launch_grp_as<W / 8, 8, DASPMM_GRP_U, TV, TB>(r, a, st);
        else return launch_grp_as<8, 4, DASPMM_GRP_U, TV, TB, 3, true>(r, a, st);  // 24 warps
    } else if constexpr (W != 128) {
        return launch_grp_narrow<W, TV, TB>(r, a, st);
    } else if constexpr (b16) {
        return launch_grp_as<16, 8, DASPMM_GRP_U16, TV, TB>(r, a, st);
    } else {  // fp8
        if (r.tiles == 1) return launch_grp_as<16, 8, DASPMM_GRP_U16, TV, TB>(r, a, st);
        return launch_grp_as<8, 16, DASPMM_GRP_U8, TV, TB>(r, a, st);
    }
}

// The walk kernel over the chunks the window kernel listed (list mode).
template <int W, typename TV, typename TB>
inline void launch_walk_list(const Resolved &r, KArgs a, cudaStream_t st)
{
    const long long resident = (long long)device_sms() * DASPMM_LEAN_MINB;
    const unsigned gx = (unsigned)std::max<long long>(
        1, std::min<long long>(((long long)a.nchunks + 7) / 8, resident));
    if (a.list_mode != 2) a.list_mode = 1;
    const unsigned gw = std::min<unsigned>(gx, (unsigned)device_sms());
    launch_pdl(k_bal_lean<W, DASPMM_LEAN_U, TV, TB, false>, dim3(gw, r.tiles), st, a);
    count_launches(1);
}

// The lean pair: for beta == 0 without Kahan rows, the window kernel (the
// worker-group form where it takes the product, else k_bal_fast) over every
// chunk and k_bal_lean over the chunks it listed; otherwise k_bal_lean over
// every chunk.  Grids: the CTAs that fit at once (chunks are handed out by
// the queue), and one CTA per SM for the listed chunks.
template <int W, typename TV, typename TB, bool K>
inline void launch_lean(const Resolved &r, KArgs a, cudaStream_t st)
{
    const long long resident = (long long)device_sms() * DASPMM_LEAN_MINB;
    const unsigned gx = (unsigned)std::max<long long>(
        1, std::min<long long>(((long long)a.nchunks + 7) / 8, resident));
    a.list_mode = 0;
    if (!K && a.beta == 0.0f) {
        if (!launch_grp<W, TV, TB>(r, a, st)) {
            if constexpr (W == 128) {
                launch_pdl(k_bal_fast<W, DASPMM_LEAN_U, TV, TB>, dim3(gx, r.tiles), st, a);
            } else {  // one queue of (tile, chunk) items
                const long long items = (long long)a.nchunks * r.tiles;
                const unsigned gi = (unsigned)std::max<long long>(
                    1, std::min<long long>((items + 7) / 8, resident));
                launch_pdl(k_bal_fast<W, DASPMM_LEAN_U, TV, TB>, dim3(gi), st, a);
            }
        }
        launch_walk_list<W, TV, TB>(r, a, st);
    } else {
        launch_pdl(k_bal_lean<W, DASPMM_LEAN_U, TV, TB, K>, dim3(gx, r.tiles), st, a);
    }
}

}  // namespace daspmm
