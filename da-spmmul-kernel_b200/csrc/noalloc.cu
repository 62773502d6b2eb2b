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

#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

namespace {

// DASPMM_NOALLOC_MAX_BYTES (daspmm.h): 16 MiB per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[DASPMM_NOALLOC_MAX_BYTES];

constexpr int kMaxDevices = 128;
std::mutex g_mu;
// Per device: the array's device address and the id of the context it was
// looked up in.  A device reset (cudaDeviceReset) ends that context; the next
// call on the device sees a new context id and looks the address up again.
struct Entry {
    unsigned long long ctx;
    void *addr;
};
Entry g_addr[kMaxDevices] = {};

using CtxGetCurrent = CUresult (*)(CUcontext *);
using CtxGetId = CUresult (*)(CUcontext, unsigned long long *);

// The id of the current device's current context (0 when it cannot be read;
// then the address is looked up on every call).  The two driver functions are
// reached through the runtime, so the library does not link libcuda itself.
unsigned long long current_context_id()
{
    static CtxGetCurrent get_current = nullptr;
    static CtxGetId get_id = nullptr;
    static bool tried = false;
    if (!tried) {
        void *f1 = nullptr, *f2 = nullptr;
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) ==
                cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<CtxGetCurrent>(f1);
            get_id = reinterpret_cast<CtxGetId>(f2);
        }
        tried = true;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || get_current(&ctx) != CUDA_SUCCESS || !ctx ||
        get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// The device address of g_noalloc_scratch on the current device.  Looked up
// with the device current, on the first call in each context of the device.
daspmm_status scratch_address(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return daspmm::cuda_fail(e);
    if (dev < 0 || dev >= kMaxDevices) return DASPMM_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_mu);
    const unsigned long long ctx = current_context_id();  // 0 before this thread's first runtime call
    if (!g_addr[dev].addr || ctx == 0 || g_addr[dev].ctx != ctx) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // makes the context current
        if (e != cudaSuccess) return daspmm::cuda_fail(e);
        g_addr[dev].addr = p;
        g_addr[dev].ctx = current_context_id();
    }
    *out = g_addr[dev].addr;
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
