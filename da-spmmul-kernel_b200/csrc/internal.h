// internal.h -- shared declarations between the translation units of
// libdaspmm.so (not installed; the public interface is include/daspmm.h).
#pragma once

#include "daspmm.h"

#include <cuda_runtime.h>
#include <stddef.h>

#include <vector>

namespace daspmm {

// A fully resolved design-space point for one problem shape.
struct Resolved {
    int alg;
    bool cm;
    int nr, nc, nnz;  // the problem it was resolved for
    int V, L, S, CF;
    int chunk, snap, nchunks;
    int block, tiles;
    int pipe;  // balanced CSR: 1 register gather, 2 TMA ring, 3 cp.async ring, 4 lean
               // gather, 5 column-major through a row-major product (transposes)
    int W;     // TMA ring: tile width in floats (32, 64, 128)
    int inner_chunk;  // pipe 5: the caller's chunk for the row-major product
    int l2_window;    // thousandths of B's lines marked L2-persisting (0 = off)
};

// SMs of the current device (148 when no device is visible).
int device_sms();

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

inline daspmm_config to_config(const Resolved &r)
{
    daspmm_config c{};
    c.alg = r.alg;
    c.vec = r.V;
    c.lanes_col = r.L;
    c.lanes_nnz = r.S;
    c.cf = r.CF;
    c.chunk = r.chunk;
    c.snap = r.snap;
    c.block = r.block;
    c.pipe = r.pipe;
    c.l2_window = r.l2_window;
    return c;
}

extern thread_local int g_last_cuda;
daspmm_status cuda_fail(cudaError_t e);

daspmm_status resolve(const daspmm_config *cfg, int layout, int nr, int nc, int nnz, int nv,
                      const void *B, const void *C, Resolved *out);
size_t workspace_bytes(const Resolved &r, int nv);
daspmm_status run_resolved(const Resolved &r, int layout, int nr, int nc, int nnz, int nv,
                           const int *rowPtr, const int *rowIdx, const int *colIdx,
                           const float *values, const float *B, float *C, float beta,
                           void *ws, size_t ws_bytes, cudaStream_t st);
// Balanced CSR: the workspace's boundary table, split-row counters, chunk
// queue heads and carry slots, and the partition launch that fills them.
struct KArgs;
void carve_balanced(const Resolved &r, void *ws, KArgs *a);
void launch_partition(const Resolved &r, int nr, int nnz, const int *rowPtr, const KArgs &a,
                      cudaStream_t st);
// carve_balanced + launch_partition on a workspace (the boundaries and the
// zeroed queue state of the balanced split).
void carve_and_partition(const Resolved &r, int nr, int nnz, const int *rowPtr, void *ws,
                         cudaStream_t st);
daspmm_status cached_workspace(size_t need, cudaStream_t st, void **out);
// A planned FP32 row-major balanced-CSR product (plan.cu): the worker-group
// window kernel alone, over a workspace whose chunk boundaries k_partition
// wrote once (the kernel leaves its queue heads and split-row counters at
// zero).  Returns false, launching nothing, when that kernel does not take
// the call (beta != 0, alignment, tile width).
// `call` counts the planned products since the boundaries were computed: a
// call's window kernel makes exactly one queue claim per chunk group, so
// each call counts its claims on from call x groups (no reset between calls).
bool run_planned(const Resolved &r, int nr, int nc, int nnz, int nv, const int *rowPtr,
                 const int *colIdx, const float *values, const float *B, float *C, void *ws,
                 unsigned long long call, cudaStream_t st);
// The boundary table and the walk list inside a balanced-CSR workspace.
void workspace_tables(const Resolved &r, void *ws, const int2 **meta, int **list);
daspmm_status cached_host_staging(size_t need, cudaStream_t st, void **out);

// Launch accounting and the optional event hook around main kernels.
void count_launches(int n);
void timer_before(cudaStream_t st);
void timer_after(cudaStream_t st);

// Batched SpMM (batch.cu), shared with the serving loop (serve.cu).
//
// A matrix is cut once into tiles (build_tiles, on the host from rowPtr):
// runs of whole rows holding at most `chunk` nonzeros plus rows (counting a
// row as one unit of work), and every row longer than `chunk` cut into pieces
// of `chunk` nonzeros.  A piece's partial sum goes to a slot; the last piece
// of a row to finish adds the row's slots in piece order and stores it, so
// results are deterministic and depend only on the matrix and `chunk`.
struct BatchTile {
    int row0, row1;   // rows [row0, row1); a piece has row1 = row0 + 1
    int k0, k1;       // piece: nonzeros [k0, k1)
    int piece;        // -1 for a run of whole rows, else the piece index
    int npieces;      // piece: pieces of the row; run: its empty rows
    int slot;         // piece: slot of piece 0 (slots slot .. slot+npieces-1)
    int cnt;          // piece: the row's counter index
};

struct TilePlan {
    std::vector<BatchTile> tiles;
    int npieces = 0;  // slots needed (x nv floats)
    int nlong = 0;    // rows cut into pieces (x column tiles counters)
};

void build_tiles(const int *rowPtr, int nr, int chunk, TilePlan *out);

// One instance as the persistent kernel sees it.  W is the instance's column
// tile width (128, 64 or 32 floats, from its own nv only).  slots holds
// npieces * nv floats, cnt nlong * col_tiles counters that start at zero and
// are left at zero by the kernel (the last piece resets its row's counter).
struct BatchInst {
    int nr, nc, nnz, nv;
    int ldb, ldc;
    int ntiles;
    int col_tiles;  // ceil(nv / W)
    int W;
    int grp;  // B and C 32-byte aligned and nv % W == 0: runs may take the group gather
    const int *rowPtr;
    const int *colIdx;
    const void *vals;
    const void *B;
    const float *bscale;
    float *C;
    const BatchTile *tiles;
    float *slots;
    int *cnt;
    float beta;
};

struct BatchItem {
    int inst, tile, ctile, pad_;
};

int batch_tile_width(int nv);
bool batch_formats_ok(int val_fmt, int b_fmt);
// Checks one instance and fills its kernel-side row except tiles / ntiles /
// slots / cnt (DASPMM_ERR_INVALID on a bad size, pointer or alignment).
daspmm_status batch_fill(const daspmm_instance &s, BatchInst *d, int wcap = 0);
daspmm_status batch_tune_chunks(const daspmm_instance *inst, int n, const int *chunks,
                                int nchunks, daspmm_config base, int reps, int *best_chunk,
                                float *best_us, void *stream);
// item table of n instances whose item counts (ntiles * col_tiles) prefix to
// d_begin[0..n].
daspmm_status batch_plan_async(const BatchInst *d_inst, const long long *d_begin, int n,
                               BatchItem *d_items, long long nitems, cudaStream_t st);
// Queue reset + one persistent launch.  wmode: the common tile width of all
// instances (128, 64, 32) or 0 when they differ; grp: with a common width,
// every instance qualifies for the worker-group gather (BatchInst::grp).
daspmm_status batch_kernel_async(int val_fmt, int b_fmt, int wmode, bool grp,
                                 const BatchInst *d_inst, const BatchItem *d_items,
                                 long long nitems, unsigned long long *d_head, cudaStream_t st);

// Autotuner (tune.cu): the cached best configuration for a shape, or the
// library's rule-of-thumb choice when nothing has been measured yet.
daspmm_status tuned_config(int layout, int nr, int nc, int nnz, int nv, daspmm_config *out);

}  // namespace daspmm
