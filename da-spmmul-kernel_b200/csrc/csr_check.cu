// csr_check.cu -- device validation of a CSR matrix.
//
// The reference trusts its inputs: the driver builds rowPtr from a sorted
// rowIdx (spmvspmm_benchmark.cu:41-76) and the kernels index B with colIdx
// unchecked (spmm.h:3-47).  A library that takes matrices from callers (and a
// server that keeps them resident for many requests) checks them once:
// rowPtr[0] == 0, rowPtr[nr] == nnz, rowPtr non-decreasing, every column in
// [0, nc), and, when asked, strictly increasing columns inside each row (the
// driver's order, spmatrix.hpp:327).
#include "daspmm.h"
#include "internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

namespace daspmm {

// One warp per row; lane 0 checks the row's pointers, all lanes its columns.
// *bad holds the smallest offending row (INT_MAX when none).
static __global__ void k_csr_check(int nr, int nc, int nnz, const int *__restrict__ rowPtr,
                                   const int *__restrict__ colIdx, int sorted, int *bad)
{
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = warp; r < nr; r += nwarps) {
        const int a = __ldg(rowPtr + r), b = __ldg(rowPtr + r + 1);
        bool ok = a >= 0 && b >= a && b <= nnz && (r != 0 || a == 0) && (r != nr - 1 || b == nnz);
        if (ok) {
            for (int k = a + lane; k < b; k += 32) {
                const int c = __ldg(colIdx + k);
                bool good = c >= 0 && c < nc;
                if (sorted && k > a) good = good && __ldg(colIdx + k - 1) < c;
                if (!good) ok = false;
            }
        }
        ok = __all_sync(0xffffffffu, ok);
        if (!ok && lane == 0) atomicMin(bad, (int)r);
    }
}

}  // namespace daspmm

using namespace daspmm;

extern "C" daspmm_status daspmm_csr_check(int nr, int nc, int nnz, const int *rowPtr,
                                          const int *colIdx, int sorted, int *bad_row,
                                          void *stream)
{
    if (bad_row) *bad_row = -1;
    if (nr < 0 || nc < 0 || nnz < 0 || (nr > 0 && !rowPtr) || (nnz > 0 && !colIdx))
        return DASPMM_ERR_INVALID;
    if (nr == 0) return nnz == 0 ? DASPMM_OK : DASPMM_ERR_BAD_MATRIX;
    cudaStream_t st = (cudaStream_t)stream;
    int *d_bad = nullptr;
    cudaError_t e = cudaMallocAsync(&d_bad, sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e);
    const int init = INT_MAX;
    int h = INT_MAX;
    e = cudaMemcpyAsync(d_bad, &init, sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const long long warps = std::min<long long>(nr, (long long)device_sms() * 64);
        const unsigned grid = (unsigned)((warps * 32 + 255) / 256);
        k_csr_check<<<grid, 256, 0, st>>>(nr, nc, nnz, rowPtr, colIdx, sorted, d_bad);
        count_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d_bad, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e);
    if (h == INT_MAX) return DASPMM_OK;
    if (bad_row) *bad_row = h;
    return DASPMM_ERR_BAD_MATRIX;
}
