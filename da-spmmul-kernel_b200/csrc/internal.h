// internal.h -- shared declarations between the translation units of
// libdaspmm.so (not installed; the public interface is include/daspmm.h).
#pragma once

#include "daspmm.h"

#include <cuda_runtime.h>
#include <stddef.h>

namespace daspmm {

// A fully resolved design-space point for one problem shape.
struct Resolved {
    int alg;
    bool cm;
    int V, L, S, CF;
    int chunk, snap, nchunks;
    int block, tiles;
    int pipe;  // balanced CSR: 1 register gather, 2 TMA ring
    int W;     // TMA ring: tile width in floats (32, 64, 128)
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
    return c;
}

extern thread_local int g_last_cuda;
daspmm_status cuda_fail(cudaError_t e);

daspmm_status resolve(const daspmm_config *cfg, int layout, int nr, int nnz, int nv,
                      const void *B, const void *C, Resolved *out);
size_t workspace_bytes(const Resolved &r, int nv);
daspmm_status run_resolved(const Resolved &r, int layout, int nr, int nc, int nnz, int nv,
                           const int *rowPtr, const int *rowIdx, const int *colIdx,
                           const float *values, const float *B, float *C, float beta,
                           void *ws, size_t ws_bytes, cudaStream_t st);
daspmm_status cached_workspace(size_t need, cudaStream_t st, void **out);
daspmm_status cached_host_staging(size_t need, cudaStream_t st, void **out);

// Launch accounting and the optional event hook around main kernels.
void count_launches(int n);
void timer_before(cudaStream_t st);
void timer_after(cudaStream_t st);

// Autotuner (tune.cu): the cached best configuration for a shape, or the
// library's rule-of-thumb choice when nothing has been measured yet.
daspmm_status tuned_config(int layout, int nr, int nc, int nnz, int nv, daspmm_config *out);

}  // namespace daspmm
