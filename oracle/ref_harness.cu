/*
 * ref_harness.cu -- C entry points into the UNMODIFIED reference
 * (ASPLOS-2022/DA-SpMMul-kernel), compiled from its own source files by
 * oracle/Makefile into oracle/_ref/libref.so.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle restatement
 * against the reference itself, and by bench.py's reference arm (the
 * reference's CPU loop timed on the host cores; its own GPU kernels and its
 * cuSPARSE helper as comparison lines).  Nothing in the shipped library links
 * it.
 *
 * The include below pulls spmvspmm_benchmark.cu from the reference tree given
 * by -I; its `main` is renamed by -Dmain=ref_main.  CUDA 12 removed three
 * cuSPARSE SpMV enum names the file uses (spmvspmm_benchmark.cu:175-178,
 * 208-211, 305-308); the Makefile maps them with -D to their CUDA 12 names.
 */
#include "spmvspmm_benchmark.cu"

#include <chrono>
#include <thread>
#include <algorithm>

extern "C" {

/* cpuSpmvReference (spmvspmm_benchmark.cu:11-39) on raw arrays. */
void ref_cpu_spmm(int layout, int nr, int nc, int nnz, int nv,
                  const int *rowPtr, const int *colIdx, const float *values,
                  const float *B, float *C)
{
    IdxArray rp(rowPtr, rowPtr + nr + 1), ci(colIdx, colIdx + nnz);
    ValArray va(values, values + nnz);
    const size_t nb = (size_t)nc * nv, nout = (size_t)nr * nv;
    ValArray in(B, B + nb), out(nout, 0.0f);
    cpuSpmvReference(layout == 1 ? DENSE_COL_MAJOR : DENSE_ROW_MAJOR, nr, nc,
                     nnz, nv, rp, ci, va, in, out);
    std::copy(out.begin(), out.end(), C);
}

/* generateCsrRowPtrArray (spmvspmm_benchmark.cu:41-76).  The reference reads
 * rowIdx[0] unconditionally, so nnz must be > 0. */
int ref_coo_to_csr(int nr, int nnz, const int *rowIdx, int *rowPtr)
{
    if (nnz <= 0) return -1;
    IdxArray ri(rowIdx, rowIdx + nnz), rp;
    generateCsrRowPtrArray(nr, rp, ri);
    std::copy(rp.begin(), rp.end(), rowPtr);
    return 0;
}

/* checkResult<host_layout, dev_layout> (spmvspmm_benchmark.cu:93-116). */
int ref_check_result(int host_layout, int dev_layout, int nrows, int ncols,
                     float *ref, float *out, float eps)
{
    if (host_layout == 0 && dev_layout == 0)
        return checkResult<DENSE_ROW_MAJOR, DENSE_ROW_MAJOR>(nrows, ncols, ref, out, eps);
    if (host_layout == 1 && dev_layout == 1)
        return checkResult<DENSE_COL_MAJOR, DENSE_COL_MAJOR>(nrows, ncols, ref, out, eps);
    if (host_layout == 0 && dev_layout == 1)
        return checkResult<DENSE_ROW_MAJOR, DENSE_COL_MAJOR>(nrows, ncols, ref, out, eps);
    return checkResult<DENSE_COL_MAJOR, DENSE_ROW_MAJOR>(nrows, ncols, ref, out, eps);
}

/* Times cpuSpmvReference on `nthreads` host threads.  The rows are split into
 * nthreads contiguous slices, each an independent sub-problem (rebased row
 * pointers, its own slice of colIdx/values and of the output) built before
 * timing; the timed region is `reps` passes of every thread calling the
 * reference function on its slice.  Returns the median wall time of one pass
 * in milliseconds. */
double ref_cpu_bench(int layout, int nr, int nc, int nnz, int nv,
                     const int *rowPtr, const int *colIdx, const float *values,
                     const float *B, int nthreads, int reps)
{
    (void)nnz;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > nr) nthreads = nr > 0 ? nr : 1;
    struct Slice { int nr, nnz; IdxArray rp, ci; ValArray va, out; };
    std::vector<Slice> sl(nthreads);
    ValArray in(B, B + (size_t)nc * nv);
    for (int t = 0; t < nthreads; ++t) {
        const int r0 = (int)((long long)nr * t / nthreads);
        const int r1 = (int)((long long)nr * (t + 1) / nthreads);
        Slice &s = sl[t];
        s.nr = r1 - r0;
        const int p0 = rowPtr[r0], p1 = rowPtr[r1];
        s.nnz = p1 - p0;
        s.rp.resize(s.nr + 1);
        for (int r = 0; r <= s.nr; ++r) s.rp[r] = rowPtr[r0 + r] - p0;
        s.ci.assign(colIdx + p0, colIdx + p1);
        s.va.assign(values + p0, values + p1);
        s.out.assign((size_t)s.nr * nv, 0.0f);
    }
    const DenseLayout lay = layout == 1 ? DENSE_COL_MAJOR : DENSE_ROW_MAJOR;
    std::vector<double> times;
    for (int it = 0; it < reps; ++it) {
        auto t0 = std::chrono::steady_clock::now();
        std::vector<std::thread> th;
        for (int t = 1; t < nthreads; ++t)
            th.emplace_back([&, t] {
                Slice &s = sl[t];
                cpuSpmvReference(lay, s.nr, nc, s.nnz, nv, s.rp, s.ci, s.va, in, s.out);
            });
        {
            Slice &s = sl[0];
            cpuSpmvReference(lay, s.nr, nc, s.nnz, nv, s.rp, s.ci, s.va, in, s.out);
        }
        for (auto &x : th) x.join();
        auto t1 = std::chrono::steady_clock::now();
        times.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
    }
    std::sort(times.begin(), times.end());
    return times.empty() ? -1.0 : times[times.size() / 2];
}

/* The reference's own GPU dispatch cudaSpmm<256,32> (spmvspmm.h:53-199) on
 * device pointers.  Returns the cudaError_t value. */
int ref_cuda_spmm(int alg, int layout, int nr, int nc, int nnz, int nv,
                  const int *rowPtr, const int *rowIdx, const int *colIdx,
                  const float *values, const float *B, float *C)
{
    return (int)cudaSpmm<256, 32>((SPMV_SPMM_ALG)alg,
                                  layout == 1 ? DENSE_COL_MAJOR : DENSE_ROW_MAJOR,
                                  nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values,
                                  B, C);
}

/* The reference's own event-timed loop, SpmvSpmmProblem::benchmark
 * (spmvspmm.h:220-243): `warmup` launches, then `reps` timed back to back on
 * stream 0; returns ms per launch (or -1 for a non-power-of-two nv). */
float ref_cuda_bench(int alg, int layout, int nr, int nc, int nnz, int nv,
                     int *rowPtr, int *rowIdx, int *colIdx, float *values,
                     float *B, float *C, int warmup, int reps)
{
    SpmvSpmmProblem prob(nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values, B, C);
    return prob.benchmark(layout == 1 ? DENSE_COL_MAJOR : DENSE_ROW_MAJOR, nv,
                          (SPMV_SPMM_ALG)alg, warmup, reps);
}

/* cuSPARSE comparison line through the reference's helper
 * (cusparse_helper.h:385-434): format 0 = CSR, 1 = COO; alg is the cuSPARSE
 * SpMM algorithm id (nv > 1).  Returns ms per call. */
float ref_cusparse_bench(int format, int layout, int nr, int nc, int nnz, int nv,
                         int *rowPtr, int *rowIdx, int *colIdx, float *values,
                         float *B, float *C, int alg, int warmup, int reps)
{
    CusparseSpmmProblem prob(nr, nc, nnz, nv, rowPtr, rowIdx, colIdx, values, B, C);
    return prob.benchmark(format == 1 ? SPARSE_FORMAT_COO : SPARSE_FORMAT_CSR,
                          layout == 1 ? DENSE_COL_MAJOR : DENSE_ROW_MAJOR, nv,
                          (cusparseSpMMAlg_t)alg, reps, warmup);
}

/* readMtx<float> (util/spmatrix.hpp:286-333), makeSymmetric included, on a
 * Matrix Market file: fills up to `cap` (row, col, value) triples in the
 * reference's output order and returns how many it produced (-1 when `cap`
 * is too small).  The reference exits the process on a missing file or a bad
 * banner, so only well-formed files may be passed. */
int ref_read_mtx(const char *path, int *nr, int *nc, int cap, int *rows, int *cols,
                 float *vals)
{
    IdxArray ri, ci;
    ValArray va;
    int nvals = 0;
    readMtx<float>(path, ri, ci, va, *nr, *nc, nvals);
    const int n = (int)ri.size();
    if (n > cap) return -1;
    for (int i = 0; i < n; ++i) {
        rows[i] = ri[i];
        cols[i] = ci[i];
        vals[i] = i < (int)va.size() ? va[i] : 0.0f;
    }
    return n;
}

} /* extern "C" */
