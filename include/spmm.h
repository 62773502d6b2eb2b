// spmm.h -- drop-in for the reference's spmm.h (ASPLOS-2022/DA-SpMMul-kernel
// spmm.h:1-512): the eight SpMM kernel templates with the same names, template
// parameters and argument lists (including the (nr, nc, nv, nnz) order of the
// two CSR col-major kernels, spmm.h:271-275 and :317-321).  Each is correct
// for ANY grid: rows / nonzero windows are grid-stride, and the dense-column
// slab comes from blockIdx.y exactly as in the reference's launches
// (spmvspmm.h:77-194).  CSR kernels overwrite C; COO kernels add into C.
//
// The library's own dispatcher (cudaSpmm in spmvspmm.h) does not use these:
// it calls libdaspmm.so, whose sm_100a kernels cover the same design space.
#pragma once
#include "spmv.h"

#ifdef __CUDACC__

// C = A B (row-major): groups of kVectorize threads per row, one column each;
// column = lane in group + blockIdx.y * kVectorize (spmm.h:3-47)
template <int kBlockSize, int kVectorize>
__global__ void spmm_csr_scalar_row_kernel(const int nr, const int nc, const int nnz,
                                           const int nv, const int *__restrict__ rowPtr,
                                           const int *__restrict__ rowIdx,
                                           const int *__restrict__ colIdx,
                                           const float *__restrict__ values,
                                           const float *__restrict__ dnInput, float *dnOutput)
{
    const int per_block = blockDim.x / kVectorize;
    const int col = (threadIdx.x % kVectorize) + blockIdx.y * kVectorize;
    if (col >= nv) return;
    for (long long r = (long long)blockIdx.x * per_block + threadIdx.x / kVectorize; r < nr;
         r += (long long)gridDim.x * per_block) {
        float acc = 0.0f;
        for (int p = __ldg(rowPtr + r); p < __ldg(rowPtr + r + 1); ++p)
            acc = fmaf(__ldg(values + p), __ldg(dnInput + (size_t)__ldg(colIdx + p) * nv + col), acc);
        dnOutput[(size_t)r * nv + col] = acc;
    }
}

// C = A B (row-major): min(nv,32)/W warps per row, each owning W columns via
// vector loads; lanes over the row's nonzeros (spmm.h:49-118)
template <int kBlockSize, typename LoadStoreType>
__global__ void spmm_csr_vector_row_kernel(const int nr, const int nc, const int nnz,
                                           const int nv, const int *__restrict__ rowPtr,
                                           const int *__restrict__ rowIdx,
                                           const int *__restrict__ colIdx,
                                           const float *__restrict__ values,
                                           const float *__restrict__ dnInput, float *dnOutput)
{
    using namespace daspmm_compat;
    constexpr int W = sizeof(LoadStoreType) / sizeof(float);
    const int lane = threadIdx.x & 31;
    const int nnv = (nv < 32 ? nv : 32) / W;
    const long long warp = gtid() >> 5, nwarps = gthreads() >> 5;
    if (nnv == 0 || nwarps < nnv) return;  // the reference uses this kernel for nv >= 8
    const int col = (int)(warp % nnv) * W + blockIdx.y * 32;
    for (long long r = warp / nnv; r < nr; r += nwarps / nnv) {
        float acc[W] = {};
        for (int p = __ldg(rowPtr + r) + lane; p < __ldg(rowPtr + r + 1); p += 32) {
            float b[W];
            ldg_float<LoadStoreType>(b, dnInput + (size_t)__ldg(colIdx + p) * nv + col);
            const float a = __ldg(values + p);
#pragma unroll
            for (int k = 0; k < W; ++k) acc[k] = fmaf(a, b[k], acc[k]);
        }
#pragma unroll
        for (int k = 0; k < W; ++k) acc[k] = daspmm_warp_sum_down(acc[k]);
        if (lane == 0) st_float<LoadStoreType>(dnOutput + (size_t)r * nv + col, acc);
    }
}

// C += A B (row-major): groups of kVectorize threads take contiguous runs of
// nonzeros, one column per thread (spmm.h:120-174)
template <int kBlockSize, int kVectorize>
__global__ void spmm_coo_scalar_row_kernel(const int nr, const int nc, const int nnz,
                                           const int nv, const int *__restrict__ rowPtr,
                                           const int *__restrict__ rowIdx,
                                           const int *__restrict__ colIdx,
                                           const float *__restrict__ values,
                                           const float *__restrict__ dnInput, float *dnOutput)
{
    const long long groups = (long long)gridDim.x * (blockDim.x / kVectorize);
    const long long g = (long long)blockIdx.x * (blockDim.x / kVectorize) + threadIdx.x / kVectorize;
    const int col = (threadIdx.x % kVectorize) + blockIdx.y * kVectorize;
    if (col >= nv) return;
    const long long per = (nnz + groups - 1) / groups;
    const long long p0 = g * per;
    if (p0 < nnz)
        daspmm_compat::coo_run_add((int)p0, (int)min((long long)nnz, p0 + per), rowIdx, colIdx,
                                   values, dnInput + col, nv, dnOutput + col, nv);
}

// C += A B (row-major): windows of 32 nonzeros, min(nv,32)/W warps across the
// columns of a 32-column slab, segmented reduction (spmm.h:176-267)
template <int kBlockSize, typename LoadStoreType>
__global__ void spmm_coo_vector_row_kernel(const int nr, const int nc, const int nnz,
                                           const int nv, const int *__restrict__ rowPtr,
                                           const int *__restrict__ rowIdx,
                                           const int *__restrict__ colIdx,
                                           const float *__restrict__ values,
                                           const float *__restrict__ dnInput, float *dnOutput)
{
    using namespace daspmm_compat;
    constexpr int W = sizeof(LoadStoreType) / sizeof(float);
    const int lane = threadIdx.x & 31;
    const int nnv = (nv < 32 ? nv : 32) / W;
    const long long warp = gtid() >> 5, nwarps = gthreads() >> 5;
    if (nnv == 0 || nwarps < nnv) return;  // the reference uses this kernel for nv >= 8
    const int col = (int)(warp % nnv) * W + blockIdx.y * 32;
    for (long long w = warp / nnv; w * 32 < nnz; w += nwarps / nnv)
        coo_window_add<W>(w * 32, nnz, lane, rowIdx, colIdx, values, dnInput + col, (size_t)nv,
                          1, dnOutput + col, (size_t)nv, 1);
}

// C = A B (col-major): one thread per row, CF columns from blockIdx.y*CF.
// Argument order (nr, nc, nv, nnz) as declared at spmm.h:271-275; neither of
// the two is read (the reference's dispatcher passes them swapped).
template <int NT, int CF>
__global__ void spmm_csr_scalar_col_kernel(const int nr, const int nc, const int nv,
                                           const int nnz, const int *__restrict__ csrRowPtr,
                                           const int *__restrict__ rowIdx,
                                           const int *__restrict__ csrCol,
                                           const float *__restrict__ csrVal,
                                           const float *__restrict__ X, float *Y)
{
    using namespace daspmm_compat;
    const float *x = X + (size_t)blockIdx.y * CF * nc;
    float *y = Y + (size_t)blockIdx.y * CF * nr;
    for (long long r = gtid(); r < nr; r += gthreads()) {
        float acc[CF] = {};
        for (int p = __ldg(csrRowPtr + r); p < __ldg(csrRowPtr + r + 1); ++p) {
            const int c = __ldg(csrCol + p);
            const float a = __ldg(csrVal + p);
#pragma unroll
            for (int k = 0; k < CF; ++k) acc[k] = fmaf(a, __ldg(x + (size_t)k * nc + c), acc[k]);
        }
#pragma unroll
        for (int k = 0; k < CF; ++k) y[(size_t)k * nr + r] = acc[k];
    }
}

// C = A B (col-major): one warp per row (spmm.h:315-367; argument order as declared)
template <int NT, int CF>
__global__ void spmm_csr_vector_col_kernel(const int nr, const int nc, const int nv,
                                           const int nnz, const int *__restrict__ csrRowPtr,
                                           const int *__restrict__ rowIdx,
                                           const int *__restrict__ csrCol,
                                           const float *__restrict__ csrVal,
                                           const float *__restrict__ X, float *Y)
{
    using namespace daspmm_compat;
    const int lane = threadIdx.x & 31;
    const float *x = X + (size_t)blockIdx.y * CF * nc;
    float *y = Y + (size_t)blockIdx.y * CF * nr;
    for (long long r = gtid() >> 5; r < nr; r += gthreads() >> 5) {
        float acc[CF] = {};
        for (int p = __ldg(csrRowPtr + r) + lane; p < __ldg(csrRowPtr + r + 1); p += 32) {
            const int c = __ldg(csrCol + p);
            const float a = __ldg(csrVal + p);
#pragma unroll
            for (int k = 0; k < CF; ++k) acc[k] = fmaf(a, __ldg(x + (size_t)k * nc + c), acc[k]);
        }
#pragma unroll
        for (int k = 0; k < CF; ++k) acc[k] = daspmm_warp_sum_down(acc[k]);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < CF; ++k) y[(size_t)k * nr + r] = acc[k];
        }
    }
}

// C += A B (col-major): contiguous nonzero runs per thread (spmm.h:370-436)
template <int NT, int CF>
__global__ void spmm_coo_scalar_col_kernel(const int nr, const int nc, const int nnz,
                                           const int nv, const int *__restrict__ rowPtr,
                                           const int *__restrict__ rowIdx,
                                           const int *__restrict__ colIdx,
                                           const float *__restrict__ values,
                                           const float *__restrict__ X, float *Y)
{
    using namespace daspmm_compat;
    const long long per = (nnz + gthreads() - 1) / gthreads();
    const long long p0 = gtid() * per;
    if (p0 >= nnz) return;
    const int p1 = (int)min((long long)nnz, p0 + per);
#pragma unroll
    for (int k = 0; k < CF; ++k)
        coo_run_add((int)p0, p1, rowIdx, colIdx, values,
                    X + (size_t)(blockIdx.y * CF + k) * nc, 1,
                    Y + (size_t)(blockIdx.y * CF + k) * nr, 1);
}

// C += A B (col-major): windows of 32 nonzeros, segmented reduction (spmm.h:438-511)
template <int NT, int CF>
__global__ void spmm_coo_vector_col_kernel(const int nr, const int nc, const int nnz,
                                           const int nv, const int *__restrict__ rowPtr,
                                           const int *__restrict__ rowIdx,
                                           const int *__restrict__ colIdx,
                                           const float *__restrict__ values,
                                           const float *__restrict__ X, float *Y)
{
    using namespace daspmm_compat;
    const int lane = threadIdx.x & 31;
    for (long long w = gtid() >> 5; w * 32 < nnz; w += gthreads() >> 5)
        coo_window_add<CF>(w * 32, nnz, lane, rowIdx, colIdx, values,
                           X + (size_t)blockIdx.y * CF * nc, 1, (size_t)nc,
                           Y + (size_t)blockIdx.y * CF * nr, 1, (size_t)nr);
}

#endif  // __CUDACC__
