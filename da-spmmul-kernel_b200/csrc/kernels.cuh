// kernels.cuh -- sm_100a SpMM/SpMV kernels (FP32) for the DA-SpMM design space.
//
// Design space (the reference's, re-expressed for B200):
//   * work split:  RB = row-balanced (a lane group per row, grid-stride),
//                  EB = nonzero-balanced (a lane group per chunk of nonzeros).
//   * reduction:   SR = the group's lanes split the dense columns and walk the
//                  nonzeros sequentially; PR = S lanes split the nonzeros and
//                  reduce with shuffles (xor tree for one row, segmented suffix
//                  scan keyed by row for EB).
//   * coarsening:  each lane owns CF vectors of V floats (V = 1/2/4, i.e. 4, 8
//                  or 16-byte accesses); a group of L lanes covers W = L*V*CF
//                  dense columns; gridDim.y walks the column tiles.
//
// Reference kernels this family replaces (ASPLOS-2022/DA-SpMMul-kernel):
//   spmm.h:3-47    spmm_csr_scalar_row_kernel   -> k_rb   (S = 1)
//   spmm.h:49-118  spmm_csr_vector_row_kernel   -> k_rb   (S > 1)
//   spmm.h:120-174 spmm_coo_scalar_row_kernel   -> k_eb_coo_sr
//   spmm.h:176-267 spmm_coo_vector_row_kernel   -> k_eb_coo_pr
//   spmm.h:269-511 the four *_col_kernel        -> the same kernels, CM = true
//   spmv.h:3-231   the four SpMV kernels        -> the same kernels, nv = 1
// The reference's COO kernels accumulate with float atomics; here a row that
// straddles chunks is written once, by a fix-up pass that adds the pieces in
// chunk order, so every result is deterministic.
//
// Layouts (spmm.h:296-310): row-major B[col*ldb + k], C[row*ldc + k];
// col-major B[k*ldb + col], C[k*ldc + row].
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace daspmm {

constexpr unsigned kFull = 0xffffffffu;

struct KArgs {
    int nr, nc, nnz, nv;
    int ldb, ldc;
    const int *__restrict__ rowPtr;
    const int *__restrict__ rowIdx;
    const int *__restrict__ colIdx;
    const float *__restrict__ vals;
    const float *__restrict__ B;
    float *C;
    float beta;         // C = A*B + beta*C; beta == 0 never reads C
    int L, S;           // lanes across dense columns, lanes across nonzeros
    int chunk;          // nonzeros per chunk (EB)
    int nchunks;
    const int2 *meta;   // balanced-CSR boundaries (k', s), nchunks + 1 entries
    float *slots;       // carries: [nchunks][2][nv] (0 = head piece, 1 = tail)
    int *own;           // ownership recording (tests): [nr][2]
    int *cnt;           // pieces arrived per split row and column tile, at the
                        // row's first chunk: [nchunks][tiles]
    unsigned int *head; // chunks handed out per column tile [tiles]
    int *list;          // chunks the fast kernel left to the walk: [0] count, then ids
    int list_mode;      // walk kernel: 0 every chunk (queue), 1 the listed ones, 2 a
                        // planned product's fixed list (window kernel: don't list)
    unsigned int head_base;  // window kernel: queue claims counted from here
    const float *bscale;  // FP8 B: per-column scales
    int kahan_min;        // rows at least this long use compensated sums
    int l2_window;        // host side: thousandths of B's lines marked L2-persisting
    size_t b_bytes;       // host side: bytes of B (the window's extent)
};

// ---------------------------------------------------------------- vectors
template <int V> struct Vec;
template <> struct Vec<1> { using T = float; };
template <> struct Vec<2> { using T = float2; };
template <> struct Vec<4> { using T = float4; };

template <int V>
__device__ __forceinline__ void ld_nc(float (&r)[V], const float *p)
{
    if constexpr (V == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
        r[0] = t.x; r[1] = t.y; r[2] = t.z; r[3] = t.w;
    } else if constexpr (V == 2) {
        const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
        r[0] = t.x; r[1] = t.y;
    } else {
        r[0] = __ldg(p);
    }
}

template <int V>
__device__ __forceinline__ void ld_plain(float (&r)[V], const float *p)
{
    if constexpr (V == 4) {
        const float4 t = *reinterpret_cast<const float4 *>(p);
        r[0] = t.x; r[1] = t.y; r[2] = t.z; r[3] = t.w;
    } else if constexpr (V == 2) {
        const float2 t = *reinterpret_cast<const float2 *>(p);
        r[0] = t.x; r[1] = t.y;
    } else {
        r[0] = *p;
    }
}

// L2-coherent load (bypasses L1): used for carries written by other CTAs.
template <int V>
__device__ __forceinline__ void ld_cg(float (&r)[V], const float *p)
{
    if constexpr (V == 4) {
        const float4 t = __ldcg(reinterpret_cast<const float4 *>(p));
        r[0] = t.x; r[1] = t.y; r[2] = t.z; r[3] = t.w;
    } else if constexpr (V == 2) {
        const float2 t = __ldcg(reinterpret_cast<const float2 *>(p));
        r[0] = t.x; r[1] = t.y;
    } else {
        r[0] = __ldcg(p);
    }
}

template <int V>
__device__ __forceinline__ void st_v(float *p, const float (&r)[V])
{
    if constexpr (V == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(r[0], r[1], r[2], r[3]);
    } else if constexpr (V == 2) {
        *reinterpret_cast<float2 *>(p) = make_float2(r[0], r[1]);
    } else {
        *p = r[0];
    }
}

// ---------------------------------------------------------------- lanes
// A "group" is G = L*S consecutive lanes of a warp.  Lane (s, l) has
// gl = s*L + l, so lanes sharing l are L apart (xor/segmented steps of L).
struct Lanes {
    int lane, G, sub, gl, s, l, base;  // base = first lane of the group
    unsigned mask;
    __device__ __forceinline__ Lanes(int L, int S)
    {
        lane = threadIdx.x & 31;
        G = L * S;
        sub = lane / G;
        base = sub * G;
        gl = lane - base;
        s = gl / L;
        l = gl - s * L;
        mask = (G == 32) ? kFull : (((1u << G) - 1u) << base);
    }
};

__device__ __forceinline__ long long group_id(int G)
{
    const int gpb = (blockDim.x >> 5) * (32 / G);
    return (long long)blockIdx.x * gpb + (threadIdx.x >> 5) * (32 / G) +
           ((threadIdx.x & 31) / G);
}

__device__ __forceinline__ long long group_count(int G)
{
    return (long long)gridDim.x * (blockDim.x >> 5) * (32 / G);
}

// Column handled by this lane for coarsening slot i of the tile.
template <int V>
__device__ __forceinline__ int lane_col(int tile_base, int i, int L, int l)
{
    return tile_base + (i * L + l) * V;
}

// B / C element addressing.
template <bool CM>
__device__ __forceinline__ const float *b_ptr(const KArgs &a, int col, int k)
{
    return CM ? a.B + (size_t)k * a.ldb + col : a.B + (size_t)col * a.ldb + k;
}
template <bool CM>
__device__ __forceinline__ float *c_ptr(const KArgs &a, int row, int k)
{
    return CM ? a.C + (size_t)k * a.ldc + row : a.C + (size_t)row * a.ldc + k;
}

// Store one output row piece: C = acc + beta*C (CM uses V == 1).
template <bool CM, int V, int CF>
__device__ __forceinline__ void store_row(const KArgs &a, int row, int tb,
                                          int L, int l, const float (&acc)[CF][V])
{
#pragma unroll
    for (int i = 0; i < CF; ++i) {
        const int k = lane_col<V>(tb, i, L, l);
        if (k < a.nv) {
            float o[V];
#pragma unroll
            for (int e = 0; e < V; ++e) o[e] = acc[i][e];
            if (a.beta != 0.0f) {
                float old[V];
                ld_plain<V>(old, c_ptr<CM>(a, row, k));
#pragma unroll
                for (int e = 0; e < V; ++e) o[e] = fmaf(a.beta, old[e], o[e]);
            }
            st_v<V>(c_ptr<CM>(a, row, k), o);
        }
    }
}

// Carry slot of chunk c: which = 0 head piece (row continued from an earlier
// chunk), 1 tail piece (row's first piece, continued by later chunks).
__device__ __forceinline__ float *slot_ptr(const KArgs &a, int c, int which, int k)
{
    return a.slots + ((size_t)c * 2 + which) * (size_t)a.nv + k;
}

template <int V, int CF>
__device__ __forceinline__ void store_slot(const KArgs &a, int c, int which,
                                           int tb, int L, int l,
                                           const float (&acc)[CF][V])
{
#pragma unroll
    for (int i = 0; i < CF; ++i) {
        const int k = lane_col<V>(tb, i, L, l);
        if (k < a.nv) st_v<V>(slot_ptr(a, c, which, k), acc[i]);
    }
}

template <int V, int CF>
__device__ __forceinline__ void zero(float (&acc)[CF][V])
{
#pragma unroll
    for (int i = 0; i < CF; ++i)
#pragma unroll
        for (int e = 0; e < V; ++e) acc[i][e] = 0.0f;
}

// Gather the CF vectors of B row `col` this lane needs.
template <bool CM, int V, int CF>
__device__ __forceinline__ void gather(const KArgs &a, int col, int tb, int L,
                                       int l, float (&b)[CF][V])
{
#pragma unroll
    for (int i = 0; i < CF; ++i) {
        const int k = lane_col<V>(tb, i, L, l);
        if (k < a.nv) {
            ld_nc<V>(b[i], b_ptr<CM>(a, col, k));
        } else {
#pragma unroll
            for (int e = 0; e < V; ++e) b[i][e] = 0.0f;
        }
    }
}

template <int V, int CF>
__device__ __forceinline__ void fma_acc(float (&acc)[CF][V], float v,
                                        const float (&b)[CF][V])
{
#pragma unroll
    for (int i = 0; i < CF; ++i)
#pragma unroll
        for (int e = 0; e < V; ++e) acc[i][e] = fmaf(v, b[i][e], acc[i][e]);
}

template <int V, int CF> constexpr int unroll_of() { return V * CF <= 4 ? 8 : (V * CF <= 8 ? 4 : 2); }

// ======================================================================
// RB: a group of G = L*S lanes per row (grid-stride over rows).
// S == 1: sequential reduction (CSR scalar); S > 1: the row's nonzeros are
// dealt round-robin to S lane sets and reduced with an xor tree (CSR vector).
// Overwrites C (beta == 0) like the reference's CSR kernels.
// ======================================================================
template <bool CM, int V, int CF>
__global__ void __launch_bounds__(256) k_rb(const KArgs a)
{
    constexpr int U = unroll_of<V, CF>();
    const int L = a.L, S = a.S;
    const Lanes ln(L, S);
    const int tb = blockIdx.y * (L * V * CF);
    const long long ng = group_count(ln.G);
    for (long long rowl = group_id(ln.G); rowl < a.nr; rowl += ng) {
        const int row = (int)rowl;
        const int p0 = __ldg(a.rowPtr + row), p1 = __ldg(a.rowPtr + row + 1);
        float acc[CF][V];
        zero<V, CF>(acc);
        int p = p0 + ln.s;
        for (; p + (U - 1) * S < p1; p += U * S) {
            int c[U];
            float v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                c[u] = __ldg(a.colIdx + p + u * S);
                v[u] = __ldg(a.vals + p + u * S);
            }
            float b[U][CF][V];
#pragma unroll
            for (int u = 0; u < U; ++u) gather<CM, V, CF>(a, c[u], tb, L, ln.l, b[u]);
#pragma unroll
            for (int u = 0; u < U; ++u) fma_acc<V, CF>(acc, v[u], b[u]);
        }
        for (; p < p1; p += S) {
            const int c = __ldg(a.colIdx + p);
            const float v = __ldg(a.vals + p);
            float b[CF][V];
            gather<CM, V, CF>(a, c, tb, L, ln.l, b);
            fma_acc<V, CF>(acc, v, b);
        }
        for (int d = L; d < ln.G; d <<= 1) {
#pragma unroll
            for (int i = 0; i < CF; ++i)
#pragma unroll
                for (int e = 0; e < V; ++e)
                    acc[i][e] += __shfl_xor_sync(ln.mask, acc[i][e], d, ln.G);
        }
        if (ln.s == 0) store_row<CM, V, CF>(a, row, tb, L, ln.l, acc);
    }
}

// ======================================================================
// EB over COO rows (rowIdx sorted): chunk c = nonzeros [c*K, min(c*K+K, nnz)).
// Rows that lie wholly inside a chunk are written directly (C = acc + beta*C;
// the reference's COO kernels use beta = 1, C += A*B).  A row that straddles
// chunks leaves one carry per chunk: the chunk holding its first nonzero
// writes the tail slot, every later chunk the head slot; k_fix_coo adds them
// in chunk order.
// ======================================================================
template <bool CM, int V, int CF, bool RECORD>
__device__ __forceinline__ void coo_finish(const KArgs &a, int c, int row, bool cont,
                                           bool ends, int tb, int L, int l,
                                           bool leader, const float (&acc)[CF][V])
{
    if constexpr (RECORD) {
        if (leader && blockIdx.y == 0) {
            atomicAdd(a.own + 2 * row + 1, 1);
            if (!cont) atomicMin(a.own + 2 * row, c);
        }
    } else {
        if (ends && !cont) store_row<CM, V, CF>(a, row, tb, L, l, acc);
        else store_slot<V, CF>(a, c, cont ? 0 : 1, tb, L, l, acc);
    }
}

template <bool CM, int V, int CF, bool RECORD>
__global__ void __launch_bounds__(256) k_eb_coo_sr(const KArgs a)
{
    constexpr int U = unroll_of<V, CF>();
    const int L = a.L;
    const Lanes ln(L, 1);
    const int G = ln.G;
    const bool wide = G >= U;            // lanes fetch a batch, then shuffle
    const int batch = wide ? G : U;
    const int tb = blockIdx.y * (L * V * CF);
    const long long ng = group_count(G);
    for (long long cl = group_id(G); cl < a.nchunks; cl += ng) {
        const int c = (int)cl;
        const long long k0 = (long long)c * a.chunk;
        const int k1 = (int)min((long long)a.nnz, k0 + a.chunk);
        int r = __ldg(a.rowIdx + k0);
        bool cont = k0 > 0 && __ldg(a.rowIdx + k0 - 1) == r;
        float acc[CF][V];
        zero<V, CF>(acc);
        for (int base = (int)k0; base < k1; base += batch) {
            const int cnt = min(batch, k1 - base);
            int my_r = 0, my_c = 0;
            float my_v = 0.0f;
            if (wide && ln.l < cnt) {
                my_r = __ldg(a.rowIdx + base + ln.l);
                if constexpr (!RECORD) {  // the recording walk gets no colIdx/values
                    my_c = __ldg(a.colIdx + base + ln.l);
                    my_v = __ldg(a.vals + base + ln.l);
                }
            }
            for (int t = 0; t < cnt; t += U) {
                int rr[U], cc[U];
                float vv[U];
                float b[U][CF][V];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (wide) {
                        const int src = (t + u) & (G - 1);
                        rr[u] = __shfl_sync(ln.mask, my_r, src, G);
                        cc[u] = __shfl_sync(ln.mask, my_c, src, G);
                        vv[u] = __shfl_sync(ln.mask, my_v, src, G);
                    } else {
                        const bool ok = t + u < cnt;
                        rr[u] = ok ? __ldg(a.rowIdx + base + t + u) : 0;
                        cc[u] = (ok && !RECORD) ? __ldg(a.colIdx + base + t + u) : 0;
                        vv[u] = (ok && !RECORD) ? __ldg(a.vals + base + t + u) : 0.0f;
                    }
                }
                if constexpr (!RECORD) {
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        if (t + u < cnt) gather<CM, V, CF>(a, cc[u], tb, L, ln.l, b[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (t + u < cnt) {
                        if (rr[u] != r) {
                            coo_finish<CM, V, CF, RECORD>(a, c, r, cont, true, tb, L, ln.l,
                                                          ln.gl == 0, acc);
                            cont = false;
                            r = rr[u];
                            zero<V, CF>(acc);
                        }
                        if constexpr (!RECORD) fma_acc<V, CF>(acc, vv[u], b[u]);
                    }
                }
            }
        }
        const bool ends = k1 >= a.nnz || __ldg(a.rowIdx + k1) != r;
        coo_finish<CM, V, CF, RECORD>(a, c, r, cont, ends, tb, L, ln.l, ln.gl == 0, acc);
    }
}

// EB with S lanes across nonzeros (COO vector): each step takes S consecutive
// nonzeros, forms the products, runs a segmented suffix scan keyed by row
// (the rows are sorted, so equal keys are contiguous), and then:
//   * the first segment joins the running row of the chunk,
//   * segments strictly inside the window are whole rows, stored directly,
//   * the last segment becomes the new running row.
template <bool CM, int V, int CF>
__global__ void __launch_bounds__(256) k_eb_coo_pr(const KArgs a)
{
    const int L = a.L, S = a.S;
    const Lanes ln(L, S);
    const int G = ln.G;
    const int tb = blockIdx.y * (L * V * CF);
    const long long ng = group_count(G);
    for (long long cl = group_id(G); cl < a.nchunks; cl += ng) {
        const int c = (int)cl;
        const long long k0 = (long long)c * a.chunk;
        const int k1 = (int)min((long long)a.nnz, k0 + a.chunk);
        int r = __ldg(a.rowIdx + k0);
        bool cont = k0 > 0 && __ldg(a.rowIdx + k0 - 1) == r;
        float run[CF][V];  // meaningful in the s == 0 lanes
        zero<V, CF>(run);
        for (int base = (int)k0; base < k1; base += S) {
            const int cnt = min(S, k1 - base);
            const int p = base + ln.s;
            const bool valid = ln.s < cnt;
            const int row = valid ? __ldg(a.rowIdx + p) : 0x7fffffff;
            float prod[CF][V];
            if (valid) {
                const int col = __ldg(a.colIdx + p);
                const float v = __ldg(a.vals + p);
                gather<CM, V, CF>(a, col, tb, L, ln.l, prod);
#pragma unroll
                for (int i = 0; i < CF; ++i)
#pragma unroll
                    for (int e = 0; e < V; ++e) prod[i][e] *= v;
            } else {
                zero<V, CF>(prod);
            }
            // segmented inclusive suffix scan over s
            for (int d = 1; d < S; d <<= 1) {
                const int orow = __shfl_down_sync(ln.mask, row, d * L, G);
                const bool take = (ln.s + d < S) && orow == row;
#pragma unroll
                for (int i = 0; i < CF; ++i)
#pragma unroll
                    for (int e = 0; e < V; ++e) {
                        const float o = __shfl_down_sync(ln.mask, prod[i][e], d * L, G);
                        if (take) prod[i][e] += o;
                    }
            }
            const int prow = __shfl_up_sync(ln.mask, row, L, G);
            const bool head = valid && (ln.s == 0 || prow != row);
            const int row0 = __shfl_sync(ln.mask, row, 0, G);
            const int rowl = __shfl_sync(ln.mask, row, (cnt - 1) * L, G);
            if (row0 != r) {  // the running row ended before this window
                if (ln.s == 0) {
                    float accv[CF][V];
#pragma unroll
                    for (int i = 0; i < CF; ++i)
#pragma unroll
                        for (int e = 0; e < V; ++e) accv[i][e] = run[i][e];
                    coo_finish<CM, V, CF, false>(a, c, r, cont, true, tb, L, ln.l, false, accv);
                }
                cont = false;
                r = row0;
                zero<V, CF>(run);
            }
            if (ln.s == 0) {
#pragma unroll
                for (int i = 0; i < CF; ++i)
#pragma unroll
                    for (int e = 0; e < V; ++e) run[i][e] += prod[i][e];
            }
            if (head && ln.s > 0 && row != rowl)  // whole row inside the window
                store_row<CM, V, CF>(a, row, tb, L, ln.l, prod);
            if (rowl != row0) {
                // the first segment is complete; the last one becomes running
                if (ln.s == 0)
                    coo_finish<CM, V, CF, false>(a, c, r, cont, true, tb, L, ln.l, false, run);
                cont = false;
                const unsigned hb = __ballot_sync(ln.mask, head && row == rowl);
                const int hl = (__ffs(hb) - 1) - ln.base;  // lane (s_h, 0) of the last head
                r = rowl;
#pragma unroll
                for (int i = 0; i < CF; ++i)
#pragma unroll
                    for (int e = 0; e < V; ++e) {
                        const float x = __shfl_sync(ln.mask, prod[i][e], hl + ln.l, G);
                        run[i][e] = x;
                    }
            }
        }
        const bool ends = k1 >= a.nnz || __ldg(a.rowIdx + k1) != r;
        if (ln.s == 0)
            coo_finish<CM, V, CF, false>(a, c, r, cont, ends, tb, L, ln.l, false, run);
    }
}

// Fix-up for the COO split: the chunk that holds the first piece of a row
// which continues past its end adds tail + later heads, in chunk order.
template <bool CM, int V, int CF>
__global__ void __launch_bounds__(256) k_fix_coo(const KArgs a)
{
    const int L = a.L;
    const Lanes ln(L, 1);
    const int tb = blockIdx.y * (L * V * CF);
    const long long ng = group_count(ln.G);
    for (long long cl = group_id(ln.G); cl + 1 < a.nchunks; cl += ng) {
        const int c = (int)cl;
        const long long k0 = (long long)c * a.chunk;
        const long long k1 = k0 + a.chunk;  // < nnz for c < nchunks - 1
        const int r = __ldg(a.rowIdx + k1 - 1);
        if (__ldg(a.rowIdx + k1) != r) continue;
        if (k0 > 0 && __ldg(a.rowIdx + k0 - 1) == r) continue;  // not its first piece
        float tot[CF][V];
#pragma unroll
        for (int i = 0; i < CF; ++i) {
            const int k = lane_col<V>(tb, i, L, ln.l);
            if (k < a.nv) ld_cg<V>(tot[i], slot_ptr(a, c, 1, k));
            else for (int e = 0; e < V; ++e) tot[i][e] = 0.0f;
        }
        for (int c2 = c + 1; c2 < a.nchunks; ++c2) {
#pragma unroll
            for (int i = 0; i < CF; ++i) {
                const int k = lane_col<V>(tb, i, L, ln.l);
                if (k < a.nv) {
                    float h[V];
                    ld_cg<V>(h, slot_ptr(a, c2, 0, k));
#pragma unroll
                    for (int e = 0; e < V; ++e) tot[i][e] += h[e];
                }
            }
            const long long e2 = min((long long)a.nnz, (long long)(c2 + 1) * a.chunk);
            if (e2 >= a.nnz || __ldg(a.rowIdx + e2) != r) break;
        }
        store_row<CM, V, CF>(a, r, tb, L, ln.l, tot);
    }
}

// ======================================================================
// Balanced CSR (EB over rowPtr, "merge" split with short-row snapping).
// k_partition writes boundary c = (k'_c, s_c) from one coalesced pass over the
// rows; k_bal walks chunk [k'_c, k'_{c+1}) with the row ends of G rows cached
// in lanes; k_fix_bal adds the carries of rows longer than the snap
// threshold that straddle chunk boundaries.
// ======================================================================
static __global__ void k_partition(int nr, int nnz, const int *__restrict__ rowPtr,
                            int chunk, int snap, int nchunks, int2 *meta, int *cnt, int tiles,
                            unsigned int *head, int *list)
{
    asm volatile("griddepcontrol.launch_dependents;");  // the gather may be scheduled now
    // launched as a programmatic dependent of the stream's previous kernel (the
    // last SpMM's walk, say): nothing is read or written before it completes
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const long long r0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r0 == 0) {
        meta[0] = make_int2(0, 0);
        meta[nchunks] = make_int2(nnz, nr);
        if (head)
            for (int t = 0; t < tiles; ++t) head[t] = 0;
        if (list) list[0] = 0;
    }
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = r0; r < nr; r += stride) {
        const int rs = __ldg(rowPtr + r), re = __ldg(rowPtr + r + 1);
        if (rs == re) continue;
        long long c = ((long long)rs + chunk - 1) / chunk;
        if (c < 1) c = 1;
        bool split = false;
        for (; c < nchunks && c * chunk < re; ++c) {
            const int k = (int)(c * chunk);
            const int kk = (k > rs && re - rs < snap) ? rs : k;
            meta[c] = make_int2(kk, (int)r);
            split |= kk > rs;
        }
        // a row split across chunks: its arrival counters (one per column
        // tile) live at its first chunk
        if (split && cnt)
            for (int t = 0; t < tiles; ++t) cnt[(size_t)(rs / chunk) * tiles + t] = 0;
    }
}

// Chunks holding pieces of a split row r (rows >= snap long are cut only at
// nominal boundaries c*chunk, so the chunk of nonzero p inside r is p/chunk).
__device__ __forceinline__ int first_chunk(int rs, int chunk) { return rs / chunk; }
__device__ __forceinline__ int last_chunk(int re, int chunk) { return (re - 1) / chunk; }

// A piece of split row `row`, already stored in its carry slot by this warp
// (tail slot in the row's first chunk, head slot in later chunks), arrives:
// it is counted at the row's first chunk and, if it is the last piece to
// arrive, the warp adds all pieces in chunk order (the first chunk's tail,
// then the heads) and stores the row: C = sum + beta*C.  VL floats per lane
// at column `col`; all lanes of the warp call it.  tiles / tile: the column
// tiles of the product and the one this piece belongs to.
template <int VL>
__device__ __forceinline__ void piece_arrive(const KArgs &a, int row, int col, int tiles,
                                             int tile)
{
    const int rs = __ldg(a.rowPtr + row), re = __ldg(a.rowPtr + row + 1);
    const int c0 = first_chunk(rs, a.chunk), c1 = last_chunk(re, a.chunk);
    __threadfence();
    __syncwarp();
    int last = 0;
    if ((threadIdx.x & 31) == 0)  // one counter per (row, column tile)
        last = atomicAdd(a.cnt + (size_t)c0 * tiles + tile, 1) == c1 - c0;
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    // every piece has arrived: the counter goes back to zero for the next call
    if ((threadIdx.x & 31) == 0) a.cnt[(size_t)c0 * tiles + tile] = 0;
    __threadfence();
    float tot[VL];
    ld_cg<VL>(tot, slot_ptr(a, c0, 1, col));
    constexpr int P = 4;  // independent carry loads in flight
    for (int cb = c0 + 1; cb <= c1; cb += P) {
        float h[P][VL];
#pragma unroll
        for (int u = 0; u < P; ++u)
            if (cb + u <= c1) ld_cg<VL>(h[u], slot_ptr(a, cb + u, 0, col));
#pragma unroll
        for (int u = 0; u < P; ++u)
            if (cb + u <= c1)
#pragma unroll
                for (int e = 0; e < VL; ++e) tot[e] += h[u][e];
    }
    float *dst = a.C + (size_t)row * a.ldc + col;
    if (a.beta != 0.0f) {
        float old[VL];
        ld_plain<VL>(old, dst);
#pragma unroll
        for (int e = 0; e < VL; ++e) tot[e] = fmaf(a.beta, old[e], tot[e]);
    }
    st_v<VL>(dst, tot);
}

// piece_arrive out of line, for kernels whose main loop needs every register
// (split rows are a small fraction of the rows).
template <int VL>
__device__ __noinline__ void piece_arrive_ool(const int *__restrict__ rowPtr, int *cnt,
                                              const float *slots, float *C, int ldc, int nv,
                                              int chunk, float beta, int row, int col,
                                              int tiles, int tile)
{
    KArgs a{};
    a.rowPtr = rowPtr;
    a.cnt = cnt;
    a.slots = const_cast<float *>(slots);
    a.C = C;
    a.ldc = ldc;
    a.nv = nv;
    a.chunk = chunk;
    a.beta = beta;
    piece_arrive<VL>(a, row, col, tiles, tile);
}

template <bool CM, int V, int CF, bool RECORD>
__device__ __forceinline__ void bal_finish(const KArgs &a, int c, int row, bool cont,
                                           bool ends, int tb, int L, int l, bool leader,
                                           const float (&acc)[CF][V])
{
    if constexpr (RECORD) {
        if (leader && blockIdx.y == 0) {
            atomicAdd(a.own + 2 * row + 1, 1);
            if (!cont) atomicMin(a.own + 2 * row, c);
        }
    } else {
        if (ends && !cont) store_row<CM, V, CF>(a, row, tb, L, l, acc);
        else store_slot<V, CF>(a, c, cont ? 0 : 1, tb, L, l, acc);
    }
}

template <bool CM, int V, int CF, bool RECORD>
__global__ void __launch_bounds__(256) k_bal(const KArgs a)
{
    constexpr int U = unroll_of<V, CF>();
    const int L = a.L;
    const Lanes ln(L, 1);
    const int G = ln.G;
    const bool wide = G >= U;
    const int batch = wide ? G : U;
    const int tb = blockIdx.y * (L * V * CF);
    const long long ng = group_count(G);
    for (long long cl = group_id(G); cl < a.nchunks; cl += ng) {
        const int c = (int)cl;
        const int2 m0 = a.meta[c], m1 = a.meta[c + 1];
        const int k0 = m0.x, k1 = m1.x, s1 = m1.y;
        int r = m0.y;
        bool cont = k0 > __ldg(a.rowPtr + r);
        // row-end cache: lane l of the group holds rowPtr[rb + 1 + l]
        int rb = r;
        int rc = __ldg(a.rowPtr + min(rb + 1 + ln.l, a.nr));
        int re = __shfl_sync(ln.mask, rc, 0, G);
        float acc[CF][V];
        zero<V, CF>(acc);
        for (int base = k0; base < k1; base += batch) {
            const int cnt = min(batch, k1 - base);
            int my_c = 0;
            float my_v = 0.0f;
            if (!RECORD && wide && ln.l < cnt) {  // the recording walk gets no colIdx/values
                my_c = __ldg(a.colIdx + base + ln.l);
                my_v = __ldg(a.vals + base + ln.l);
            }
            for (int t = 0; t < cnt; t += U) {
                int cc[U];
                float vv[U];
                float b[U][CF][V];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (wide) {
                        const int src = (t + u) & (G - 1);
                        cc[u] = __shfl_sync(ln.mask, my_c, src, G);
                        vv[u] = __shfl_sync(ln.mask, my_v, src, G);
                    } else {
                        const bool ok = t + u < cnt && !RECORD;
                        cc[u] = ok ? __ldg(a.colIdx + base + t + u) : 0;
                        vv[u] = ok ? __ldg(a.vals + base + t + u) : 0.0f;
                    }
                }
                if constexpr (!RECORD) {
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        if (t + u < cnt) gather<CM, V, CF>(a, cc[u], tb, L, ln.l, b[u]);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (t + u < cnt) {
                        const int p = base + t + u;
                        while (p >= re) {
                            bal_finish<CM, V, CF, RECORD>(a, c, r, cont, true, tb, L, ln.l,
                                                          ln.gl == 0, acc);
                            cont = false;
                            zero<V, CF>(acc);
                            ++r;
                            if (r - rb >= G) {
                                rb = r;
                                rc = __ldg(a.rowPtr + min(rb + 1 + ln.l, a.nr));
                            }
                            re = __shfl_sync(ln.mask, rc, r - rb, G);
                        }
                        if constexpr (!RECORD) fma_acc<V, CF>(acc, vv[u], b[u]);
                    }
                }
            }
        }
        // rows that end at or before k1 (incl. trailing empty rows), then the
        // first piece of row s1 if it started inside this chunk
        while (r < s1) {
            bal_finish<CM, V, CF, RECORD>(a, c, r, cont, true, tb, L, ln.l, ln.gl == 0, acc);
            cont = false;
            zero<V, CF>(acc);
            ++r;
        }
        if (r < a.nr && r == s1 && __ldg(a.rowPtr + r) < k1)
            bal_finish<CM, V, CF, RECORD>(a, c, r, cont, false, tb, L, ln.l, ln.gl == 0, acc);
    }
}

template <bool CM, int V, int CF>
__global__ void __launch_bounds__(256) k_fix_bal(const KArgs a)
{
    const int L = a.L;
    const Lanes ln(L, 1);
    const int tb = blockIdx.y * (L * V * CF);
    const long long ng = group_count(ln.G);
    for (long long cl = group_id(ln.G); cl + 1 < a.nchunks; cl += ng) {
        const int c = (int)cl;
        const int k0 = a.meta[c].x;
        const int2 m1 = a.meta[c + 1];
        const int k1 = m1.x, r = m1.y;
        const int rs = __ldg(a.rowPtr + r);
        if (!(rs < k1 && rs >= k0)) continue;  // no first piece of row r here
        const int re = __ldg(a.rowPtr + r + 1);
        float tot[CF][V];
#pragma unroll
        for (int i = 0; i < CF; ++i) {
            const int k = lane_col<V>(tb, i, L, ln.l);
            if (k < a.nv) ld_cg<V>(tot[i], slot_ptr(a, c, 1, k));
            else for (int e = 0; e < V; ++e) tot[i][e] = 0.0f;
        }
        for (int c2 = c + 1; c2 < a.nchunks; ++c2) {
#pragma unroll
            for (int i = 0; i < CF; ++i) {
                const int k = lane_col<V>(tb, i, L, ln.l);
                if (k < a.nv) {
                    float h[V];
                    ld_cg<V>(h, slot_ptr(a, c2, 0, k));
#pragma unroll
                    for (int e = 0; e < V; ++e) tot[i][e] += h[e];
                }
            }
            if (re <= a.meta[c2 + 1].x) break;
        }
        store_row<CM, V, CF>(a, r, tb, L, ln.l, tot);
    }
}

// C = beta * C over an nr x nv block (used before COO accumulation when
// beta != 1, since COO never visits rows without nonzeros).
// dst (Cn x R) = transpose of src (R x Cn) + beta * dst, both row-major: 32 x 32
// tiles through shared memory (reads and writes are 128-byte rows), the grid
// striding over tiles.  beta == 0 never reads dst.
static __global__ void __launch_bounds__(256) k_transpose(const float *__restrict__ src,
                                                          long long R, long long Cn,
                                                          float *__restrict__ dst, float beta)
{
    __shared__ float tile[32][33];
    const long long tx = (Cn + 31) / 32, ty = (R + 31) / 32;
    for (long long t = blockIdx.x; t < tx * ty; t += gridDim.x) {
        const long long r0 = (t / tx) * 32, c0 = (t % tx) * 32;
        for (int i = threadIdx.y; i < 32; i += 8) {
            const long long r = r0 + i, c = c0 + threadIdx.x;
            if (r < R && c < Cn) tile[i][threadIdx.x] = __ldg(src + r * Cn + c);
        }
        __syncthreads();
        for (int i = threadIdx.y; i < 32; i += 8) {
            const long long c = c0 + i, r = r0 + threadIdx.x;  // dst row c, column r
            if (c < Cn && r < R) {
                float *d = dst + c * R + r;
                const float v = tile[threadIdx.x][i];
                *d = beta == 0.0f ? v : fmaf(beta, *d, v);
            }
        }
        __syncthreads();
    }
}

static __global__ void k_scale(float *C, size_t n, float beta)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        C[i] = beta == 0.0f ? 0.0f : beta * C[i];
}

// rowPtr[r] = number of nonzeros with row < r, from sorted COO rows: every
// nonzero p whose row differs from its predecessor's fills the pointers of
// the rows in between (empty rows included).  Bit-exact with
// generateCsrRowPtrArray (spmvspmm_benchmark.cu:41-76).
static __global__ void k_coo_to_csr(int nr, int nnz, const int *__restrict__ rowIdx, int *rowPtr)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p > nnz) return;
    const int prev = p == 0 ? -1 : __ldg(rowIdx + p - 1);
    const int cur = p == nnz ? nr : __ldg(rowIdx + p);
    for (int r = prev + 1; r <= cur && r <= nr; ++r) rowPtr[r] = (int)p;
}

// Ownership recording buffers (tests): owner = INT_MAX / pieces = 0, then
// unowned rows back to -1 after the walk.
static __global__ void k_own_init(int *own, int nr)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nr) { own[2 * r] = 0x7fffffff; own[2 * r + 1] = 0; }
}
static __global__ void k_own_fini(int *own, int nr)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nr && own[2 * r] == 0x7fffffff) own[2 * r] = -1;
}

}  // namespace daspmm
