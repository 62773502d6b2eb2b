// noalloc.cu -- daspmm_spmm_noalloc: the balanced-CSR SpMM for callers that
// cannot allocate device memory.
//
// Some callers can't call cudaMalloc at all: a library loaded as a plugin into
// a host application whose own allocator owns the whole device (a framework
// memory pool, a fixed per-plugin budget), or a loop that must not pay the
// device-wide synchronisation that cudaMalloc/cudaFree imply.  daspmm_spmm
// would allocate its workspace on first use, and daspmm_spmm_ex needs one from
// the caller; this entry point needs neither.  Its scratch -- the chunk
// boundary table and the carry slots of rows split across chunks -- lives in
// the fixed array below, which every GPU that loads the library holds until
// the process exits.
#include "internal.h"

#include <cuda_runtime.h>

#include <mutex>

namespace {

// DASPMM_NOALLOC_MAX_BYTES (daspmm.h): 16 MiB per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[DASPMM_NOALLOC_MAX_BYTES];

constexpr int kMaxDevices = 128;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// The device address of g_noalloc_scratch on the current device.  Looked up
// once per device (the first call on that device), with the device current.
daspmm_status scratch_address(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return daspmm::cuda_fail(e);
    if (dev < 0 || dev >= kMaxDevices) return DASPMM_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return daspmm::cuda_fail(e);
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return DASPMM_OK;
}

}  // namespace

extern "C" daspmm_status daspmm_spmm_noalloc(int layout, int nr, int nc, int nnz, int nv,
                                             const int *rowPtr, const int *colIdx,
                                             const float *values, const float *B, float *C,
                                             float beta, void *stream)
{
    daspmm_config cfg{};
    cfg.alg = DASPMM_ALG_CSR_BALANCED;
    // column-major: the direct gather (the transposing path would need
    // scratch for copies of B and C)
    if (layout == DASPMM_COL_MAJOR) cfg.pipe = 1;
    daspmm::Resolved r;
    daspmm_status s = daspmm::resolve(&cfg, layout, nr, nc, nnz, nv, B, C, &r);
    if (s != DASPMM_OK) return s;
    // Too large for the fixed scratch: refuse before touching the device.
    if (daspmm::workspace_bytes(r, nv) > (size_t)DASPMM_NOALLOC_MAX_BYTES)
        return DASPMM_ERR_WORKSPACE;
    void *scratch = nullptr;
    s = scratch_address(&scratch);
    if (s != DASPMM_OK) return s;
    // Every scratch entry the kernels read (boundary table, carry slots) is
    // written earlier in the same call, so nothing needs clearing between calls.
    return daspmm::run_resolved(r, layout, nr, nc, nnz, nv, rowPtr, nullptr, colIdx, values, B,
                                C, beta, scratch, (size_t)DASPMM_NOALLOC_MAX_BYTES,
                                (cudaStream_t)stream);
}
