// Test harness: launches the drop-in kernel templates of include/spmm.h and
// include/spmv.h with the grids the reference's dispatcher computes
// (ASPLOS-2022/DA-SpMMul-kernel spmvspmm.h:72-197), so the tests can check
// that each template is correct under exactly those launches.
#include "spmvspmm.h"

namespace {
constexpr int kB = 256, kW = 32;

template <typename K>
int go(K kernel, dim3 grid, int block, int nr, int nc, int nnz, int nv, const int *rp,
       const int *ri, const int *ci, const float *va, const float *B, float *C)
{
    if (grid.x == 0 || grid.y == 0) return (int)cudaErrorInvalidConfiguration;
    kernel<<<grid, block>>>(nr, nc, nnz, nv, rp, ri, ci, va, B, C);
    return (int)cudaGetLastError();
}
}  // namespace

extern "C" int launch_ref_grid(int alg, int layout, int nr, int nc, int nnz, int nv,
                               const int *rp, const int *ri, const int *ci, const float *va,
                               const float *B, float *C)
{
#define ARGS nr, nc, nnz, nv, rp, ri, ci, va, B, C
    if (layout == DENSE_ROW_MAJOR) {
        if (alg == ALG_CSR_SCALAR || alg == ALG_COO_SCALAR) {
            const int bx = nv < 32 ? nv : 32, by = kB / bx;
            const dim3 g(DIV_UP(nr, by), nv > 32 ? nv / 32 : 1);
            const bool coo = alg == ALG_COO_SCALAR;
            switch (nv) {
            case 1: return coo ? go(spmv_coo_scalar_kernel<kB>, g, kB, ARGS)
                               : go(spmv_csr_scalar_kernel<kB>, g, kB, ARGS);
            case 2: return coo ? go(spmm_coo_scalar_row_kernel<kB, 2>, g, kB, ARGS)
                               : go(spmm_csr_scalar_row_kernel<kB, 2>, g, kB, ARGS);
            case 4: return coo ? go(spmm_coo_scalar_row_kernel<kB, 4>, g, kB, ARGS)
                               : go(spmm_csr_scalar_row_kernel<kB, 4>, g, kB, ARGS);
            case 8: return coo ? go(spmm_coo_scalar_row_kernel<kB, 8>, g, kB, ARGS)
                               : go(spmm_csr_scalar_row_kernel<kB, 8>, g, kB, ARGS);
            case 16: return coo ? go(spmm_coo_scalar_row_kernel<kB, 16>, g, kB, ARGS)
                                : go(spmm_csr_scalar_row_kernel<kB, 16>, g, kB, ARGS);
            default: return coo ? go(spmm_coo_scalar_row_kernel<kB, 32>, g, kB, ARGS)
                                : go(spmm_csr_scalar_row_kernel<kB, 32>, g, kB, ARGS);
            }
        }
        const int elems = nv > 4 ? 4 : nv;
        const int warps = (DIV_UP(nnz, kW) < nr ? DIV_UP(nnz, kW) : nr) * ((nv < 32 ? nv : 32) / elems);
        const dim3 g(warps / (kB / kW), nv > 32 ? nv / 32 : 1);
        const bool coo = alg == ALG_COO_VECTOR;
        switch (nv) {
        case 1: return coo ? go(spmv_coo_vector_kernel<kB, float>, g, kB, ARGS)
                           : go(spmv_csr_vector_kernel<kB, float>, g, kB, ARGS);
        case 2: return coo ? go(spmv_coo_vector_kernel<kB, float2>, g, kB, ARGS)
                           : go(spmv_csr_vector_kernel<kB, float2>, g, kB, ARGS);
        case 4: return coo ? go(spmv_coo_vector_kernel<kB, float4>, g, kB, ARGS)
                           : go(spmv_csr_vector_kernel<kB, float4>, g, kB, ARGS);
        default: return coo ? go(spmm_coo_vector_row_kernel<kB, float4>, g, kB, ARGS)
                            : go(spmm_csr_vector_row_kernel<kB, float4>, g, kB, ARGS);
        }
    }
    if (alg == ALG_CSR_SCALAR || alg == ALG_COO_SCALAR) {
        const bool coo = alg == ALG_COO_SCALAR;
        if (nv == 1)
            return coo ? go(spmv_coo_scalar_kernel<kB>, dim3(DIV_UP(nr, kB)), kB, ARGS)
                       : go(spmv_csr_scalar_kernel<kB>, dim3(DIV_UP(nr, kB)), kB, ARGS);
        return coo ? go(spmm_coo_scalar_col_kernel<kB, 1>, dim3(DIV_UP(nr, kB), nv), kB, ARGS)
                   : go(spmm_csr_scalar_col_kernel<kB, 1>, dim3(DIV_UP(nr, kB), nv), kB, ARGS);
    }
    const int warps = (DIV_UP(nnz, kW) < nr ? DIV_UP(nnz, kW) : nr) * nv;
    const bool coo = alg == ALG_COO_VECTOR;
    if (nv == 1)
        return coo ? go(spmv_coo_vector_kernel<kB, float>, dim3(warps / (kB / kW)), kB, ARGS)
                   : go(spmv_csr_vector_kernel<kB, float>, dim3(warps / (kB / kW)), kB, ARGS);
    return coo ? go(spmm_coo_vector_col_kernel<kB, 1>, dim3(DIV_UP(nnz, kB / 32), nv), kB, ARGS)
               : go(spmm_csr_vector_col_kernel<kB, 1>, dim3(DIV_UP(nr, kB / 32), nv), kB, ARGS);
#undef ARGS
}
