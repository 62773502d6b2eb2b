/*
 * oracle.h -- CPU restatement of the reference's host-side arithmetic for the
 * SpMM/SpMV path, plus the partition tables the CUDA kernels must reproduce
 * bit for bit.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline and reference legs of bench.py may load this library, and only
 * as the checker (or, in the reference leg, to build that leg's inputs).
 * The shipped library (libdaspmm.so) never links or calls it.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the ASPLOS-2022/DA-SpMMul-kernel source tree).
 */
#ifndef DASPMM_ORACLE_H
#define DASPMM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Dense layouts: same values as enum DenseLayout (helper.h:261-264). */
#define OR_ROW_MAJOR 0
#define OR_COL_MAJOR 1

/* COO row indices (sorted by row) -> CSR row pointer rowPtr[nr+1].
 * Restates generateCsrRowPtrArray (spmvspmm_benchmark.cu:41-76): rowPtr[r] is
 * the position of the first nonzero of row r; empty leading, middle and
 * trailing rows get the position of the next nonempty row (or nnz).  The
 * reference reads rowIdx[0] unguarded (:44); here nnz == 0 is defined and
 * yields an all-zero rowPtr.  Returns 0, or -1 if rowIdx is not sorted or out
 * of range. */
int or_coo_to_csr_rowptr(int nr, int nnz, const int *rowIdx, int *rowPtr);

/* FP32 host SpMM in the reference's exact loop order and rounding
 * (cpuSpmvReference, spmvspmm_benchmark.cu:11-39).  Row-major: per row a
 * zeroed accumulator vector, nonzeros outer, dense columns inner (:27-37).
 * Col-major: dense column outer, row, nonzero (:13-25).  Compiled without FMA
 * contraction so every step is one fp32 multiply then one fp32 add, as in the
 * reference built for x86-64.
 * B: RM nc x nv (B[col*nv+k]); CM (B[k*nc+col]).  C likewise with nr. */
void or_spmm_f32(int layout, int nr, int nc, int nnz, int nv,
                 const int *rowPtr, const int *colIdx, const float *values,
                 const float *B, float *C);

/* FP64 oracle of the same product, used for error statements.  Optionally
 * also writes absC[i] = sum_p |a_p| * |b_p| (the condition scale of each
 * output element), in the layout of C.  absC may be NULL. */
void or_spmm_f64(int layout, int nr, int nc, int nnz, int nv,
                 const int *rowPtr, const int *colIdx, const float *values,
                 const float *B, double *C, double *absC);

/* Same as or_spmm_f64 but the inputs are double (used after quantising to
 * BF16/FP16/FP8 on the host). */
void or_spmm_f64d(int layout, int nr, int nc, int nnz, int nv,
                  const int *rowPtr, const int *colIdx, const double *values,
                  const double *B, double *C, double *absC);

/* checkResult (spmvspmm_benchmark.cu:93-116): absolute |out-ref| > eps fails;
 * stops at the first failing element when first_only is nonzero.  host_layout
 * and dev_layout give the layout of ref and out.  Returns 1 when passed; on
 * failure writes the first failing (i, j) to *bad_i, *bad_j (may be NULL). */
int or_check_result(int host_layout, int dev_layout, int nrows, int ncols,
                    const float *ref, const float *out, float eps,
                    int first_only, int *bad_i, int *bad_j);

/* calcMaxNv (spmvspmm_benchmark.cu:78-90): the largest power of two <= maxnv
 * whose dense input and output (nc + nr) * nv * dtype_size fit, with the
 * sparse matrix, in mem_bytes. */
int or_calc_max_nv(int nr, int nc, int nnz, size_t mem_bytes, int dtype_size,
                   int maxnv);

/* ---- Partition arithmetic (no reference counterpart; the reference's
 * binary_search_segment_number sketch at helper.h:283-321 is commented out).
 * These define the row/nonzero ownership the CUDA kernels implement. ---- */

/* upper_bound(rowPtr[0..nr], k) - 1: the last row r with rowPtr[r] <= k. */
int or_row_of(const int *rowPtr, int nr, int k);

/* Number of nonzero-balanced chunks: max(1, ceil(nnz / chunk)). */
int or_num_chunks(int nnz, int chunk);

/* Balanced-CSR split table.  For every boundary c in [0, nchunks]:
 *   meta[2c]   = k'_c, the snapped first nonzero of chunk c,
 *   meta[2c+1] = s_c,  the row containing k'_c.
 * Nominal boundary k = c*chunk; s = or_row_of(k); when k falls strictly
 * inside row s and that row has fewer than `snap` nonzeros, the boundary moves
 * down to the row's first nonzero (short rows are never split).  Boundary 0 is
 * (0, 0) and boundary nchunks is (nnz, nr).  meta has 2*(nchunks+1) ints. */
void or_balanced_partition(int nr, int nnz, const int *rowPtr, int chunk,
                           int snap, int *meta);

/* Output-row ownership for the balanced-CSR split, derived by walking every
 * chunk exactly as the kernels do.  For every row r:
 *   owner[2r]   = chunk that writes C[r] (directly, or in the fix-up pass),
 *   owner[2r+1] = number of chunks that hold a piece of row r (1 = the row is
 *                 written directly by its chunk; >1 = split, written by the
 *                 fix-up of the owner chunk; 0 = empty row, written directly).
 * Returns 0, or -1 if the walk finds an inconsistency. */
int or_balanced_ownership(int nr, int nnz, const int *rowPtr, int chunk,
                          int snap, int *owner);

/* Ownership for the nonzero-balanced COO split (chunk c = [c*K, (c+1)*K)):
 * same encoding as above; rows without nonzeros get owner -1, pieces 0
 * (COO algorithms never touch them). */
int or_coo_ownership(int nr, int nnz, const int *rowIdx, int chunk, int *owner);

/* ---- Reduced-precision storage formats (round to nearest even). ---- */
uint16_t or_f32_to_bf16(float x);
float or_bf16_to_f32(uint16_t h);
uint16_t or_f32_to_f16(float x);
float or_f16_to_f32(uint16_t h);
/* FP8 E4M3 (OCP/NVIDIA "e4m3fn"): bias 7, max finite 448, no infinities,
 * saturating conversion of finite values (satfinite). */
uint8_t or_f32_to_e4m3(float x);
float or_e4m3_to_f32(uint8_t v);

/* Bulk helpers: convert n floats (q is 16-bit or 8-bit storage). */
void or_quantize(int fmt, size_t n, const float *x, void *q);
void or_dequantize(int fmt, size_t n, const void *q, double *x);
/* fmt ids: 0 = f32, 1 = bf16, 2 = f16, 3 = e4m3 (same as daspmm.h) */

/* ---- Seeded synthetic workloads: restatements of libdaspmm's generators
 * (daspmm_gen_uniform / _powerlaw / _dense), so that the benchmark's
 * reference arm builds its inputs without the product library.  Same
 * arguments and outputs; 0 on success, -1 on bad arguments. ---- */
int or_gen_uniform(int nr, int nc, int per_row, uint64_t seed, int *rowPtr, int *colIdx,
                   float *values);
int or_gen_powerlaw(int nr, int nc, double alpha, double shift, int dmin, int dmax,
                    double mean_scale, uint64_t seed, int *rowPtr, int *colIdx,
                    float *values, long long *nnz_out);
void or_gen_dense(size_t n, uint64_t seed, float lo, float hi, float *out);

#ifdef __cplusplus
}
#endif
#endif
