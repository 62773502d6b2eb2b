// gather_tma.cuh -- balanced-CSR SpMM with a TMA-fed shared-memory ring.
//
// The register-gather kernel (k_bal) is latency-bound: each warp has at most
// one unrolled group of B-row loads in flight and its registers cap the
// number of resident warps.  Here every warp owns a ring of NS stages in
// shared memory; a stage holds the B-tile rows (W floats each) of Q nonzeros
// plus their values.  One lane per nonzero issues a 1-D bulk copy
// (cp.async.bulk: one instruction moves a whole W*4-byte row) that completes
// on the stage's mbarrier; the warp consumes stage i while stages i+1..i+NS-1
// are in flight, and refills stage i with block i+NS as soon as it is read.
// Column indices and values of block i+NS are loaded into registers before
// stage i is awaited, so their latency hides behind the wait.
//
// Same chunk boundaries (k_partition), walk, ownership and carry slots as
// k_bal, so k_fix_bal finishes rows split across chunks unchanged.
// Row-major only; needs nv % W == 0 and a 16-byte aligned B (every copied
// row segment then starts on a 16-byte boundary and stays inside B).
#pragma once

#include "kernels.cuh"
#include "tma.cuh"

namespace daspmm {

template <int W, int NS>
struct TmaRing {
    static constexpr int kRowBytes = W * 4;
    static constexpr int Q = 4096 / kRowBytes;        // nonzeros per stage
    static constexpr int kTileBytes = NS * 4096;
    static constexpr int kValBytes = NS * Q * 4;
    static constexpr int kBarOff = (kTileBytes + kValBytes + 7) & ~7;
    static constexpr int kWarpBytes = (kBarOff + NS * 8 + 127) & ~127;
    static constexpr int kWarps = 4;                  // warps per CTA
    static constexpr int kCtaBytes = kWarps * kWarpBytes;
};

// MODE 0: one lane per nonzero issues a bulk copy of the whole row segment
// (TMA engine), completion on the stage mbarrier.  MODE 1: the warp copies
// the row segments itself with 16-byte cp.async (W/4 lanes per row, 128/W
// rows per instruction), one commit group per stage.
template <int W, int NS, int MODE>
__global__ void __launch_bounds__(128) k_bal_tma(const KArgs a)
{
    using R = TmaRing<W, NS>;
    constexpr int VL = W / 32;  // floats per lane
    constexpr int Q = R::Q;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *wbase = smem + warp * R::kWarpBytes;
    float *tiles = reinterpret_cast<float *>(wbase);
    float *svals = reinterpret_cast<float *>(wbase + R::kTileBytes);
    const uint32_t bar0 = smem_addr(wbase + R::kBarOff);
    if (lane == 0)
        for (int s = 0; s < NS; ++s) mbar_init(bar0 + 8 * s, 1);
    mbar_init_fence();
    __syncwarp();

    const uint64_t pol_keep = policy_evict_last();   // B rows: reused across warps
    const uint64_t pol_once = policy_evict_first();  // index/value streams
    const int tb = blockIdx.y * W;
    const float *Bt = a.B + tb;
    const long long nwarps = (long long)gridDim.x * R::kWarps;
    long long g = 0;  // blocks this warp has consumed: stage = g % NS, parity = (g / NS) & 1

    for (long long cl = (long long)blockIdx.x * R::kWarps + warp; cl < a.nchunks; cl += nwarps) {
        const int c = (int)cl;
        const int2 m0 = a.meta[c], m1 = a.meta[c + 1];
        const int k0 = m0.x, k1 = m1.x, s1 = m1.y;
        int r = m0.y;
        bool cont = k0 > __ldg(a.rowPtr + r);
        const int nb = (k1 - k0 + Q - 1) / Q;

        // issue block i of this chunk into its stage (col/val of slot q held by lane q)
        auto issue = [&](int i, int col, float val) {
            const int p0 = k0 + i * Q;
            const int cnt = i < nb ? min(Q, k1 - p0) : 0;
            const int s = (int)((g + i) % NS);
            if (lane < cnt) svals[s * Q + lane] = val;
            if constexpr (MODE == 0) {
                if (cnt == 0) return;
                const uint32_t bar = bar0 + 8 * s;
                if (lane < cnt) {
                    fence_proxy_async_smem();
                    bulk_g2s(smem_addr(tiles + (size_t)(s * Q + lane) * W),
                             Bt + (size_t)col * a.ldb, R::kRowBytes, bar, pol_keep);
                }
                if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)(cnt * R::kRowBytes));
            } else {
                constexpr int LR = W / 4;       // lanes per row segment (16 bytes each)
                constexpr int RPI = 32 / LR;    // row segments per warp instruction
                const int part = lane % LR, sub = lane / LR;
#pragma unroll
                for (int t = 0; t < Q / RPI; ++t) {
                    const int q = t * RPI + sub;
                    const int cq = __shfl_sync(kFull, col, q);
                    if (q < cnt)
                        cp_async16(smem_addr(tiles + (size_t)(s * Q + q) * W + part * 4),
                                   Bt + (size_t)cq * a.ldb + part * 4, pol_keep);
                }
                cp_async_commit();  // one group per stage, empty ones included
            }
        };

        // Column indices / values run 2*NS blocks ahead of consumption: lane q
        // keeps those of slot q of blocks i+NS .. i+2NS-1 in a FIFO (fc, fv).
        auto load_cv = [&](int j, int &col, float &val) {
            const int p = k0 + j * Q + lane;
            const bool ok = j < nb && lane < Q && p < k1;
            col = ok ? ld_hint_s32(a.colIdx + p, pol_once) : 0;
            val = ok ? ld_hint_f32(a.vals + p, pol_once) : 0.0f;
        };
        int fc[NS];
        float fv[NS];
        {
            int pc[NS];
            float pv[NS];
#pragma unroll
            for (int u = 0; u < NS; ++u) load_cv(u, pc[u], pv[u]);
#pragma unroll
            for (int u = 0; u < NS; ++u) load_cv(NS + u, fc[u], fv[u]);
#pragma unroll
            for (int u = 0; u < NS; ++u)
                if (MODE == 1 || u < nb) issue(u, pc[u], pv[u]);
        }

        // row-end cache (lane l holds rowPtr[rb + 1 + l]) and its prefetch
        int rb = r;
        int rc = __ldg(a.rowPtr + min(rb + 1 + lane, a.nr));
        int rn = __ldg(a.rowPtr + min(rb + 33 + lane, a.nr));
        int re = __shfl_sync(kFull, rc, 0);
        float acc[VL];
#pragma unroll
        for (int e = 0; e < VL; ++e) acc[e] = 0.0f;

        auto emit = [&](int row, bool ends) {
            float *dst;
            bool direct = ends && !cont;
            if (direct) dst = a.C + (size_t)row * a.ldc + tb + lane * VL;
            else dst = slot_ptr(a, c, cont ? 0 : 1, tb + lane * VL);
            float o[VL];
#pragma unroll
            for (int e = 0; e < VL; ++e) o[e] = acc[e];
            if (direct && a.beta != 0.0f) {
                float old[VL];
                ld_plain<VL>(old, dst);
#pragma unroll
                for (int e = 0; e < VL; ++e) o[e] = fmaf(a.beta, old[e], o[e]);
            }
            st_hint<VL>(dst, o, pol_once);
#pragma unroll
            for (int e = 0; e < VL; ++e) acc[e] = 0.0f;
            cont = false;
        };
        auto next_row = [&]() {
            ++r;
            if (r - rb >= 32) {
                rb += 32;
                rc = rn;
                rn = __ldg(a.rowPtr + min(rb + 33 + lane, a.nr));
            }
            re = __shfl_sync(kFull, rc, r - rb);
        };

        bool alive = true;
        int i = 0;
        for (int i0 = 0; i0 < nb && alive; i0 += NS) {
#pragma unroll
            for (int u = 0; u < NS; ++u) {
                i = i0 + u;
                if (i >= nb) break;
                const int s = (int)((g + i) % NS);
                if constexpr (MODE == 0) {
                    // every lane polls; the warp goes on only if all lanes saw the phase
                    const bool ok = mbar_wait(bar0 + 8 * s, (uint32_t)(((g + i) / NS) & 1));
                    if (!__all_sync(kFull, ok)) {
                        alive = false;
                        break;
                    }
                } else {
                    cp_async_wait<NS - 1>();  // this stage's group (always NS groups pending)
                    __syncwarp();             // every lane's copies visible to the warp
                }
                const int p0 = k0 + i * Q;
                const int cnt = min(Q, k1 - p0);
                const float *st = tiles + (size_t)s * Q * W + lane * VL;
                const float *sv = svals + s * Q;
                for (int q = 0; q < cnt; ++q) {
                    const int p = p0 + q;
                    while (p >= re) {
                        emit(r, true);
                        next_row();
                    }
                    const float v = sv[q];
                    float b[VL];
                    ld_plain<VL>(b, st + q * W);
#pragma unroll
                    for (int e = 0; e < VL; ++e) acc[e] = fmaf(v, b[e], acc[e]);
                }
                __syncwarp();
                if (MODE == 1 || i + NS < nb) issue(i + NS, fc[u], fv[u]);
                load_cv(i + 2 * NS, fc[u], fv[u]);
            }
        }
        if (!alive) {
            // a wait expired: let this warp's copies in flight land (bounded), then stop
            for (int k = i; k < min(nb, i + NS); ++k)
                mbar_wait(bar0 + 8 * (int)((g + k) % NS), (uint32_t)(((g + k) / NS) & 1));
            return;
        }
        // (MODE 1: the NS groups still pending here belong to blocks past the
        // chunk's end and are empty; the next chunk's waits count past them.)
        g += nb;
        // rows ending at or before k1 (trailing empty rows included), then the
        // first piece of row s1 if it started inside this chunk
        while (r < s1) {
            emit(r, true);
            ++r;
        }
        if (r < a.nr && r == s1 && __ldg(a.rowPtr + r) < k1) emit(r, false);
    }
}

}  // namespace daspmm
