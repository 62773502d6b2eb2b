// mixed.cu -- mixed-precision SpMM (BF16 / FP16 storage, FP8 E4M3 B with
// per-column scales, FP32 accumulation, optional Kahan rows) and the device
// quantizers that produce its inputs.  No counterpart in the reference, whose
// kernels are FP32 only (spmm.h:17-18); this extends that value/B type.
#include "gather_lean.cuh"
#include "internal.h"
#include "kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>

namespace daspmm {

template <int W, typename TV, typename TB, bool K>
static void launch_mixed_w(const Resolved &r, const KArgs &a, cudaStream_t st)
{
    launch_lean<W, TV, TB, K>(r, a, st);
}

template <typename TV, typename TB>
static void launch_mixed(const Resolved &r, const KArgs &a, bool kahan, cudaStream_t st)
{
#define DASPMM_MW(w)                                                                        \
    if (r.W == w) {                                                                         \
        if (kahan) launch_mixed_w<w, TV, TB, true>(r, a, st);                               \
        else launch_mixed_w<w, TV, TB, false>(r, a, st);                                   \
        return;                                                                             \
    }
    DASPMM_MW(128) DASPMM_MW(64) DASPMM_MW(32)
#undef DASPMM_MW
}

static size_t fmt_bytes(int f)
{
    return f == DASPMM_F32 ? 4 : (f == DASPMM_E4M3 ? 1 : 2);
}

template <typename TQ>
__device__ __forceinline__ TQ quant(float x);
template <> __device__ __forceinline__ bf16 quant<bf16>(float x) { return __float2bfloat16_rn(x); }
template <> __device__ __forceinline__ fp16 quant<fp16>(float x) { return __float2half_rn(x); }
template <> __device__ __forceinline__ fp8 quant<fp8>(float x)
{
    fp8 q;
    q.__x = __nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
    return q;
}

// q[i] = round(x[i] / scale[i % ncols]) (scale may be null: 1)
template <typename TQ>
static __global__ void k_quantize(const float *__restrict__ x, TQ *q, size_t n,
                                  const float *__restrict__ scale, int ncols)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        float v = x[i];
        if (scale) v = v / scale[i % (size_t)ncols];
        q[i] = quant<TQ>(v);
    }
}

// amax[k] = max_i |B[i, k]| as float bits (non-negative floats order as
// unsigned integers, so an integer max is exact and order-independent)
static __global__ void k_colmax(const float *__restrict__ B, int nrows, int ncols,
                                unsigned *amax)
{
    const int col = blockIdx.x * 32 + (threadIdx.x & 31);
    if (col >= ncols) return;
    unsigned m = 0;
    for (long long i = (long long)blockIdx.y * (blockDim.x / 32) + (threadIdx.x >> 5); i < nrows;
         i += (long long)gridDim.y * (blockDim.x / 32))
        m = max(m, __float_as_uint(fabsf(B[(size_t)i * ncols + col])));
    atomicMax(amax + col, m);
}

static __global__ void k_zero_u32(unsigned *p, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = 0;
}

// scale[k] = amax[k] / 448 (the largest finite E4M3), 1 for an all-zero column
static __global__ void k_scale_finish(unsigned *amax_bits, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float m = __uint_as_float(amax_bits[i]);
    reinterpret_cast<float *>(amax_bits)[i] = m > 0.0f ? m / 448.0f : 1.0f;
}

}  // namespace daspmm

using namespace daspmm;

extern "C" {

daspmm_status daspmm_spmm_mixed(const daspmm_config *cfg_in, int layout, int nr, int nc, int nnz,
                                int nv, const int *rowPtr, const int *colIdx,
                                const void *values, int val_fmt, const void *B, int b_fmt,
                                const float *b_scales, float *C, float beta, int kahan_min,
                                void *workspace, size_t ws_bytes, void *stream)
{
    if (layout != DASPMM_ROW_MAJOR) return DASPMM_ERR_UNSUPPORTED;
    if (val_fmt < DASPMM_F32 || val_fmt > DASPMM_F16) return DASPMM_ERR_UNSUPPORTED;
    if (b_fmt < DASPMM_F32 || b_fmt > DASPMM_E4M3) return DASPMM_ERR_INVALID;
    if (b_fmt == DASPMM_E4M3 && !b_scales) return DASPMM_ERR_INVALID;
    const bool combo = (val_fmt == DASPMM_F32 && b_fmt == DASPMM_F32) ||
                       (val_fmt == DASPMM_BF16 && b_fmt == DASPMM_BF16) ||
                       (val_fmt == DASPMM_F16 && b_fmt == DASPMM_F16) ||
                       (val_fmt == DASPMM_F32 && b_fmt == DASPMM_E4M3) ||
                       (val_fmt == DASPMM_BF16 && b_fmt == DASPMM_E4M3);
    if (!combo) return DASPMM_ERR_UNSUPPORTED;
    daspmm_config cfg = cfg_in ? *cfg_in : daspmm_config{};
    cfg.alg = DASPMM_ALG_CSR_BALANCED;
    if (cfg.pipe && cfg.pipe != 4) return DASPMM_ERR_UNSUPPORTED;
    cfg.pipe = 4;
    // measured: reduced-precision B (the 16-lane group kernel) runs best, like
    // FP32, at 96 nonzeros per chunk for one 128-column tile and at 128 for
    // wider products (BF16 N = 128: 71.3 against 74.2 us; E4M3 64.6 against
    // 65.4).  Never more chunks than the FP32 default, so a workspace sized
    // for it still suffices.
    if (!cfg.chunk) cfg.chunk = nv == 128 ? 96 : 128;
    Resolved r;
    daspmm_status s = resolve(&cfg, layout, nr, nc, nnz, nv, nullptr, C, &r);
    if (s != DASPMM_OK) return s;
    if (r.pipe != 4) return DASPMM_ERR_UNSUPPORTED;  // needs nv % 32 == 0
    const int VL = r.W / 32;
    if (B && ((uintptr_t)B % (VL * fmt_bytes(b_fmt)))) return DASPMM_ERR_INVALID;
    if (nr == 0) return DASPMM_OK;
    if (!B || !C || !rowPtr || (nnz > 0 && (!colIdx || !values))) return DASPMM_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t need = workspace_bytes(r, nv);
    if (!workspace) {
        s = cached_workspace(need, st, &workspace);
        if (s != DASPMM_OK) return s;
        ws_bytes = need;
    }
    if (need > ws_bytes) return DASPMM_ERR_WORKSPACE;

    KArgs a{};
    a.nr = nr; a.nc = nc; a.nnz = nnz; a.nv = nv;
    a.ldb = nv; a.ldc = nv;
    a.rowPtr = rowPtr; a.colIdx = colIdx;
    a.vals = reinterpret_cast<const float *>(values);
    a.B = reinterpret_cast<const float *>(B);
    a.C = C; a.beta = beta;
    a.L = r.L; a.S = 1; a.chunk = r.chunk; a.nchunks = r.nchunks;
    a.bscale = b_scales;
    a.kahan_min = kahan_min > 0 ? kahan_min : 0x7fffffff;
    a.l2_window = r.l2_window;
    a.b_bytes = (size_t)fmt_bytes(b_fmt) * nc * nv;
    carve_balanced(r, workspace, &a);
    launch_partition(r, nr, nnz, rowPtr, a, st);
    timer_before(st);  // the optional timer brackets the main kernel
    const bool kahan = kahan_min > 0;
    if (val_fmt == DASPMM_F32 && b_fmt == DASPMM_F32) launch_mixed<float, float>(r, a, kahan, st);
    else if (val_fmt == DASPMM_BF16 && b_fmt == DASPMM_BF16) launch_mixed<bf16, bf16>(r, a, kahan, st);
    else if (val_fmt == DASPMM_F16) launch_mixed<fp16, fp16>(r, a, kahan, st);
    else if (val_fmt == DASPMM_F32) launch_mixed<float, fp8>(r, a, kahan, st);
    else launch_mixed<bf16, fp8>(r, a, kahan, st);
    timer_after(st);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

daspmm_status daspmm_quantize(int fmt, size_t n, const float *x, void *q, const float *col_scales,
                              int ncols, void *stream)
{
    if (n == 0) return DASPMM_OK;
    if (!x || !q || (col_scales && ncols <= 0)) return DASPMM_ERR_INVALID;
    const unsigned g = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 64);
    cudaStream_t st = (cudaStream_t)stream;
    switch (fmt) {
    case DASPMM_BF16: k_quantize<bf16><<<g, 256, 0, st>>>(x, (bf16 *)q, n, col_scales, ncols); break;
    case DASPMM_F16: k_quantize<fp16><<<g, 256, 0, st>>>(x, (fp16 *)q, n, col_scales, ncols); break;
    case DASPMM_E4M3: k_quantize<fp8><<<g, 256, 0, st>>>(x, (fp8 *)q, n, col_scales, ncols); break;
    default: return DASPMM_ERR_UNSUPPORTED;
    }
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

daspmm_status daspmm_e4m3_scales(int nrows, int ncols, const float *B, float *scales, void *stream)
{
    if (nrows < 0 || ncols <= 0 || !scales || (nrows > 0 && !B)) return DASPMM_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned *bits = reinterpret_cast<unsigned *>(scales);
    k_zero_u32<<<(ncols + 255) / 256, 256, 0, st>>>(bits, ncols);
    if (nrows > 0) {
        const unsigned gy = (unsigned)std::min<long long>(((long long)nrows + 7) / 8, 1024);
        k_colmax<<<dim3((ncols + 31) / 32, gy), 256, 0, st>>>(B, nrows, ncols, bits);
    }
    k_scale_finish<<<(ncols + 255) / 256, 256, 0, st>>>(bits, ncols);
    count_launches(nrows > 0 ? 3 : 2);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DASPMM_OK : cuda_fail(e);
}

}  // extern "C"
