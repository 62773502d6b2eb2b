// spmvspmm.h -- drop-in for the reference's spmvspmm.h (ASPLOS-2022/
// DA-SpMMul-kernel spmvspmm.h:1-273): SPMV_SPMM_ALG, SpmvSpmmProblem and
// cudaSpmm<kBlockSize, kWarpSize> with the same names, values and signatures.
// cudaSpmm forwards to libdaspmm.so (daspmm_compat_spmm in daspmm.h), whose
// sm_100a kernels replace the reference's twelve; the kernel templates of
// spmm.h / spmv.h stay available for code that launches them itself.
//
// Link with -ldaspmm (da-spmmul-kernel_b200/libdaspmm.so).
#pragma once

#include "spmm.h"
#include "spmv.h"
#include "daspmm.h"

#include <cuda_profiler_api.h>
#include <iostream>

// spmvspmm.h:5-10 (same enumerator values as DASPMM_ALG_*)
enum SPMV_SPMM_ALG { ALG_CSR_SCALAR = 0, ALG_CSR_VECTOR = 1, ALG_COO_SCALAR = 2, ALG_COO_VECTOR = 3 };

// spmvspmm.h:53-199.  CSR algorithms overwrite dnOutput, COO algorithms add
// into it; launches go to the legacy default stream; the cudaError_t of the
// launch is returned.  kBlockSize / kWarpSize are accepted for source
// compatibility; the library picks its own CTA shapes for sm_100a.
template <int kBlockSize = 256, int kWarpSize = 32>
cudaError_t cudaSpmm(SPMV_SPMM_ALG kAlg, DenseLayout layout, const int nr, const int nc,
                     const int nnz, const int nv, const int *rowPtr, const int *rowIdx,
                     const int *colIdx, const float *values, const float *dnInput,
                     float *dnOutput)
{
    return (cudaError_t)daspmm_compat_spmm((int)kAlg, (int)layout, nr, nc, nnz, nv, rowPtr,
                                           rowIdx, colIdx, values, dnInput, dnOutput);
}

// spmvspmm.h:13-50: a non-owning view of device buffers.
struct SpmvSpmmProblem {
    int nr, nc, nnz, maxNv;
    int *rowPtr, *rowIdx, *colIdx;
    float *values, *dnInput, *dnOutput;

    SpmvSpmmProblem(int nr, int nc, int nnz, int maxNv, int *rowPtr, int *rowIdx, int *colIdx,
                    float *values, float *dnInput, float *dnOutput)
        : nr(nr), nc(nc), nnz(nnz), maxNv(maxNv), rowPtr(rowPtr), rowIdx(rowIdx),
          colIdx(colIdx), values(values), dnInput(dnInput), dnOutput(dnOutput)
    {
    }

    // spmvspmm.h:202-218: power-of-two nv check (print and return), then one
    // call; a CUDA error ends the process as in the reference (CUDA_CHECK).
    void run(DenseLayout layout, int nv, SPMV_SPMM_ALG alg)
    {
        if ((nv & (nv - 1)) != 0) {
            std::cerr << "nv must be power of 2, less than 32. Got nv = " << nv << std::endl;
            return;
        }
        CUDA_CHECK(cudaSpmm<>(alg, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values,
                              dnInput, dnOutput));
    }

    // spmvspmm.h:220-243: warm-up, then repeatIters back-to-back calls timed
    // with events on stream 0; ms per call, or -1 for a bad nv.
    float benchmark(DenseLayout layout, int nv, SPMV_SPMM_ALG alg, int warmupIters = 5,
                    int repeatIters = 50)
    {
        if ((nv & (nv - 1)) != 0) {
            std::cerr << "nv must be power of 2, less than 32. Got nv = " << nv << std::endl;
            return -1;
        }
        cudaError_t status = cudaSuccess;
        hgpu::GpuTimer timer;
        for (int i = 0; i < warmupIters; ++i)
            status = cudaSpmm<>(alg, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values,
                                dnInput, dnOutput);
        CUDA_CHECK(status);
        CUDA_CHECK(cudaDeviceSynchronize());
        timer.start();
        for (int i = 0; i < repeatIters; ++i)
            status = cudaSpmm<>(alg, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values,
                                dnInput, dnOutput);
        timer.stop();
        CUDA_CHECK(status);
        return timer.elapsed_msecs() / (float)repeatIters;
    }

    // spmvspmm.h:245-273: warm-up, then one call between cudaProfilerStart/Stop.
    void dry_run(DenseLayout layout, int nv, SPMV_SPMM_ALG alg, int warmupIters = 0)
    {
        if ((nv & (nv - 1)) != 0 || nv > 32) {
            std::cerr << "nv must be power of 2, less than 32. Got nv = " << nv << std::endl;
            return;
        }
        cudaError_t status = cudaSuccess;
        for (int i = 0; i < warmupIters; ++i)
            status = cudaSpmm<>(alg, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values,
                                dnInput, dnOutput);
        CUDA_CHECK(status);
        CUDA_CHECK(cudaDeviceSynchronize());
#ifndef FLAG_GPGPUSIM
        cudaProfilerStart();
#endif
        status = cudaSpmm<>(alg, layout, nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values, dnInput,
                            dnOutput);
#ifndef FLAG_GPGPUSIM
        cudaProfilerStop();
#endif
        CUDA_CHECK(status);
    }
};
