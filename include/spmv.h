// spmv.h -- drop-in for the reference's spmv.h (ASPLOS-2022/DA-SpMMul-kernel
// spmv.h:1-231): the four SpMV kernel templates with the same names, template
// parameters and argument lists, so code that launches them directly still
// compiles and runs.  They are written to be correct for ANY grid (grid-stride
// over rows / nonzero windows), including every grid the reference's
// dispatcher computes.  CSR kernels overwrite y; COO kernels add into y.
//
// The library's own dispatcher (cudaSpmm in spmvspmm.h) does not use these:
// it calls libdaspmm.so, whose sm_100a kernels cover the same design space.
#pragma once
#include "helper.h"

#ifdef __CUDACC__

namespace daspmm_compat {

__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ long long gthreads() { return (long long)gridDim.x * blockDim.x; }

// Sequential run over nonzeros [p, e) of sorted COO rows: one atomic add per
// row segment into out[row * stride + col_off].
__device__ __forceinline__ void coo_run_add(int p, int e, const int *__restrict__ rowIdx,
                                            const int *__restrict__ colIdx,
                                            const float *__restrict__ values,
                                            const float *__restrict__ x, int x_stride,
                                            float *out, int out_stride)
{
    if (p >= e) return;
    int cur = __ldg(rowIdx + p);
    float acc = 0.0f;
    for (; p < e; ++p) {
        const int r = __ldg(rowIdx + p);
        if (r != cur) {
            atomicAdd(out + (size_t)cur * out_stride, acc);
            acc = 0.0f;
            cur = r;
        }
        acc = fmaf(__ldg(values + p), __ldg(x + (size_t)__ldg(colIdx + p) * x_stride), acc);
    }
    atomicAdd(out + (size_t)cur * out_stride, acc);
}

// One warp over 32 consecutive nonzeros [base, base+32) of sorted COO rows:
// products of `W` columns per lane, segmented suffix sum, atomics at segment
// heads.  Out-of-range lanes carry key INT_MAX and zero.
template <int W>
__device__ __forceinline__ void coo_window_add(long long base, int nnz, int lane,
                                               const int *__restrict__ rowIdx,
                                               const int *__restrict__ colIdx,
                                               const float *__restrict__ values,
                                               const float *__restrict__ x, size_t x_row,
                                               size_t x_col, float *out, size_t o_row,
                                               size_t o_col)
{
    const long long p = base + lane;
    const bool in = p < nnz;
    const int row = in ? __ldg(rowIdx + p) : 0x7fffffff;
    float v[W];
    if (in) {
        const float a = __ldg(values + p);
        const int c = __ldg(colIdx + p);
#pragma unroll
        for (int k = 0; k < W; ++k) v[k] = a * __ldg(x + (size_t)c * x_row + k * x_col);
    } else {
#pragma unroll
        for (int k = 0; k < W; ++k) v[k] = 0.0f;
    }
#pragma unroll
    for (int k = 0; k < W; ++k) v[k] = daspmm_warp_seg_suffix(v[k], row, lane);
    const int prev = __shfl_up_sync(FULLMASK, row, 1);
    if (in && (lane == 0 || prev != row)) {
#pragma unroll
        for (int k = 0; k < W; ++k) atomicAdd(out + (size_t)row * o_row + k * o_col, v[k]);
    }
}

}  // namespace daspmm_compat

// y = A x, one thread per row (spmv.h:3-39)
template <int kCtaSize>
__global__ void spmv_csr_scalar_kernel(const int nr, const int nc, const int nnz, const int nv,
                                       const int *__restrict__ rowPtr,
                                       const int *__restrict__ rowIdx,
                                       const int *__restrict__ colIdx,
                                       const float *__restrict__ values,
                                       const float *__restrict__ dnInput, float *dnOutput)
{
    using namespace daspmm_compat;
    for (long long r = gtid(); r < nr; r += gthreads()) {
        float acc = 0.0f;
        for (int p = __ldg(rowPtr + r); p < __ldg(rowPtr + r + 1); ++p)
            acc = fmaf(__ldg(values + p), __ldg(dnInput + __ldg(colIdx + p)), acc);
        dnOutput[r] = acc;
    }
}

// y += A x, each thread a contiguous run of DIV_UP(nnz, threads) nonzeros (spmv.h:41-89)
template <int kCtaSize>
__global__ void spmv_coo_scalar_kernel(const int nr, const int nc, const int nnz, const int nv,
                                       const int *__restrict__ rowPtr,
                                       const int *__restrict__ rowIdx,
                                       const int *__restrict__ colIdx,
                                       const float *__restrict__ values,
                                       const float *__restrict__ dnInput, float *dnOutput)
{
    using namespace daspmm_compat;
    const long long per = (nnz + gthreads() - 1) / gthreads();
    const long long p0 = gtid() * per;
    if (p0 < nnz)
        coo_run_add((int)p0, (int)min((long long)nnz, p0 + per), rowIdx, colIdx, values, dnInput, 1,
                    dnOutput, 1);
}

// y = A X for nv = sizeof(T)/4 in {1, 2, 4}: one warp per row, lanes over the
// row's nonzeros, vector loads of B rows (spmv.h:91-147)
template <int kCtaSize, typename LoadStoreType>
__global__ void spmv_csr_vector_kernel(const int nr, const int nc, const int nnz, const int nv,
                                       const int *__restrict__ rowPtr,
                                       const int *__restrict__ rowIdx,
                                       const int *__restrict__ colIdx,
                                       const float *__restrict__ values,
                                       const float *__restrict__ dnInput, float *dnOutput)
{
    using namespace daspmm_compat;
    constexpr int W = sizeof(LoadStoreType) / sizeof(float);
    const int lane = threadIdx.x & 31;
    for (long long r = gtid() >> 5; r < nr; r += gthreads() >> 5) {
        float acc[W] = {};
        for (int p = __ldg(rowPtr + r) + lane; p < __ldg(rowPtr + r + 1); p += 32) {
            float b[W];
            ldg_float<LoadStoreType>(b, dnInput + (size_t)__ldg(colIdx + p) * nv);
            const float a = __ldg(values + p);
#pragma unroll
            for (int k = 0; k < W; ++k) acc[k] = fmaf(a, b[k], acc[k]);
        }
#pragma unroll
        for (int k = 0; k < W; ++k) acc[k] = daspmm_warp_sum_down(acc[k]);
        if (lane == 0) st_float<LoadStoreType>(dnOutput + (size_t)r * nv, acc);
    }
}

// y += A X, one warp per window of 32 nonzeros, segmented reduction (spmv.h:149-231)
template <int kBlockSize, typename LoadStoreType>
__global__ void spmv_coo_vector_kernel(const int nr, const int nc, const int nnz, const int nv,
                                       const int *__restrict__ rowPtr,
                                       const int *__restrict__ rowIdx,
                                       const int *__restrict__ colIdx,
                                       const float *__restrict__ values,
                                       const float *__restrict__ dnInput, float *dnOutput)
{
    using namespace daspmm_compat;
    constexpr int W = sizeof(LoadStoreType) / sizeof(float);
    const int lane = threadIdx.x & 31;
    for (long long w = gtid() >> 5; w * 32 < nnz; w += gthreads() >> 5)
        coo_window_add<W>(w * 32, nnz, lane, rowIdx, colIdx, values, dnInput, (size_t)nv, 1,
                          dnOutput, (size_t)nv, 1);
}

#endif  // __CUDACC__
