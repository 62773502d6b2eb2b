/*
 * daspmm.h -- C ABI of the B200 (sm_100a) SpMM/SpMV library libdaspmm.so.
 *
 * Plain C: pointers, sizes and status codes; no CUDA or C++ types.  Device
 * pointers are raw CUDA device addresses owned by the caller; `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream, which is
 * what the reference uses for every launch, helper.h:176,181).
 *
 * Sparse matrix A: nr x nc with nnz nonzeros, int32 indices, sorted by
 * (row, col).  CSR algorithms read rowPtr[nr+1]; COO algorithms read
 * rowIdx[nnz]; both read colIdx[nnz] and values[nnz] (the reference's driver
 * supplies both arrays over the same colIdx/values,
 * spmvspmm_benchmark.cu:367-376).  Dense B is nc x nv and C is nr x nv, both
 * row-major (B[col*nv+k]) or both col-major (B[k*nc+col]), as in
 * spmm.h:296-310.
 *
 * No function here exits the process or prints; every failure is a status.
 */
#ifndef DASPMM_H
#define DASPMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define DASPMM_ABI_VERSION 2

typedef enum daspmm_status {
    DASPMM_OK = 0,
    DASPMM_ERR_INVALID = 1,      /* bad argument: sizes, null pointer, layout, nv */
    DASPMM_ERR_UNSUPPORTED = 2,  /* combination of algorithm/layout/config not provided */
    DASPMM_ERR_CUDA = 3,         /* a CUDA call failed; see daspmm_last_cuda_error() */
    DASPMM_ERR_NOMEM = 4,        /* device allocation failed */
    DASPMM_ERR_WORKSPACE = 5,    /* caller workspace smaller than required */
    DASPMM_ERR_TIMEOUT = 6,      /* a bounded wait expired */
    DASPMM_ERR_BUDGET = 7,       /* request exceeds the memory budget (serving) */
    DASPMM_ERR_CANCELLED = 8,    /* request cancelled (serving) */
    DASPMM_ERR_BAD_MATRIX = 9    /* validation failed: rowPtr/rowIdx/colIdx malformed */
} daspmm_status;

/* Algorithm ids 0..3 have the values of enum SPMV_SPMM_ALG
 * (spmvspmm.h:5-10) and the reference's semantics: CSR algorithms overwrite C
 * (C = A*B), COO algorithms accumulate (C += A*B) -- see beta below. */
enum {
    DASPMM_ALG_CSR_SCALAR = 0,   /* row-balanced, sequential reduction   (SR_RB) */
    DASPMM_ALG_CSR_VECTOR = 1,   /* row-balanced, warp-parallel reduction (PR_RB) */
    DASPMM_ALG_COO_SCALAR = 2,   /* nonzero-balanced, sequential          (SR_EB) */
    DASPMM_ALG_COO_VECTOR = 3,   /* nonzero-balanced, segmented parallel   (PR_EB) */
    DASPMM_ALG_CSR_BALANCED = 4, /* nonzero-balanced over CSR with short-row snapping */
    DASPMM_ALG_AUTO = 5          /* autotuned choice among the above (CSR semantics) */
};

/* Dense layouts: values of enum DenseLayout (helper.h:261-264). */
enum { DASPMM_ROW_MAJOR = 0, DASPMM_COL_MAJOR = 1 };

/* Storage formats for the mixed-precision entry points. */
enum { DASPMM_F32 = 0, DASPMM_BF16 = 1, DASPMM_F16 = 2, DASPMM_E4M3 = 3 };

/* A point of the design space.  Zero fields take the library default for the
 * problem shape. */
typedef struct daspmm_config {
    int alg;        /* DASPMM_ALG_* (0..4) */
    int vec;        /* floats per vector access: 1, 2 or 4 (16-byte loads) */
    int lanes_col;  /* L: lanes splitting the dense columns (power of two <= 32) */
    int lanes_nnz;  /* S: lanes splitting the nonzeros (power of two, L*S <= 32) */
    int cf;         /* column-coarsening factor: vectors per lane (1, 2; CM 1..8) */
    int chunk;      /* nonzeros per chunk for the nonzero-balanced splits */
    int snap;       /* balanced CSR: rows shorter than this are never split */
    int block;      /* threads per CTA: 128 or 256 */
    int pipe;       /* balanced CSR, row-major: 1 = register gather; a shared-memory
                       ring fed by 2 = TMA bulk copies, 3 = 16-byte cp.async;
                       4 = lean register gather at high occupancy (2..4 need
                       nv % 32 == 0 and 16-byte aligned B and C).  Column-major:
                       1 = direct gather, 5 = B transposed to row-major, the
                       row-major product, C transposed back (the default from
                       nv >= 4; A read once for all columns).
                       0 = the library's choice */
    int l2_window;  /* balanced CSR, row-major window and walk kernels: 0 = off;
                       1..1000 = an L2 access-policy window over B on the main
                       kernel's launch, that many thousandths of its lines
                       marked persisting (the rest streaming).  Has an effect
                       only with a persisting L2 set-aside
                       (daspmm_l2_set_aside).  Results do not depend on it. */
} daspmm_config;

/* ---- FP32 SpMM ---------------------------------------------------------
 * C = A*B + beta*C.  beta == 0 never reads C.  For the COO algorithms a beta
 * other than 1 first scales all of C (rows without nonzeros included).
 * Uses a workspace the library keeps per (device, stream); the call that first
 * needs a larger one synchronises the stream and allocates (so it must not be
 * the first call inside a stream capture).
 * Replaces: cudaSpmm<kBlockSize,kWarpSize>(alg, layout, nr, nc, nnz, nv,
 * rowPtr, rowIdx, colIdx, values, dnInput, dnOutput) (spmvspmm.h:53-199),
 * which has beta fixed by the algorithm. */
daspmm_status daspmm_spmm(int alg, int layout, int nr, int nc, int nnz, int nv,
                          const int *rowPtr, const int *rowIdx, const int *colIdx,
                          const float *values, const float *B, float *C,
                          float beta, void *stream);

/* Same with an explicit design-space point and caller-owned workspace of
 * ws_bytes (>= daspmm_workspace_bytes(...)); workspace == NULL falls back to
 * the library's per-stream workspace.  No counterpart in the reference (its
 * template parameters kBlockSize/kWarpSize are fixed at 256/32). */
daspmm_status daspmm_spmm_ex(const daspmm_config *cfg, int layout, int nr, int nc,
                             int nnz, int nv, const int *rowPtr, const int *rowIdx,
                             const int *colIdx, const float *values, const float *B,
                             float *C, float beta, void *workspace, size_t ws_bytes,
                             void *stream);

/* Workspace bytes daspmm_spmm_ex needs for this configuration and shape
 * (pipe 5 holds row-major copies of B and C, so nc matters). */
size_t daspmm_workspace_bytes(const daspmm_config *cfg, int layout, int nr, int nc, int nnz,
                              int nv);

/* Fill *out with the configuration the library would use for this shape
 * (the defaults; or the autotuner's cached choice for DASPMM_ALG_AUTO once
 * daspmm_autotune has run for the fingerprint). */
daspmm_status daspmm_default_config(int alg, int layout, int nr, int nc, int nnz,
                                    int nv, daspmm_config *out);

/* ---- Autotuner ---------------------------------------------------------
 * No counterpart in the reference: its caller picks alg (spmvspmm.h:57-58).
 * A fingerprint of a problem: shape, storage and row-length quantiles
 * (computed on the device from rowPtr; quantiles are the upper edges of
 * power-of-two length buckets, capped at the maximum). */
typedef struct daspmm_fingerprint {
    int layout, nv, dtype, nr, nnz;
    int p50, p90, p99, max_row;
} daspmm_fingerprint;

daspmm_status daspmm_fingerprint_of(int layout, int nr, int nnz, int nv, int dtype,
                                    const int *rowPtr, void *stream, daspmm_fingerprint *out);

/* Times the design-space candidates that apply (reps calls each, after two
 * warm-up calls; C is overwritten) and caches the fastest under the
 * fingerprint; DASPMM_ALG_AUTO then uses it for the same (layout, nv, nr, nnz).
 * rowIdx may be NULL (COO candidates are then skipped).  Returns the choice
 * and its time per call in microseconds. */
daspmm_status daspmm_autotune(int layout, int nr, int nc, int nnz, int nv, const int *rowPtr,
                              const int *rowIdx, const int *colIdx, const float *values,
                              const float *B, float *C, int reps, daspmm_config *best,
                              float *best_us, void *stream);
/* The cache as a text file (one line per fingerprint), and back. */
daspmm_status daspmm_tune_save(const char *path);
daspmm_status daspmm_tune_load(const char *path);
void daspmm_tune_clear(void);

/* ---- Drop-in for the reference's dispatcher ------------------------------
 * Exactly cudaSpmm<256,32> (spmvspmm.h:53-199): CSR algorithms overwrite C,
 * COO algorithms add into C, the legacy default stream, and the return value
 * is a cudaError_t (0 = cudaSuccess; cudaErrorInvalidValue = 1 for bad
 * arguments).  Any nv >= 1 is accepted (the reference's power-of-two check
 * lives in SpmvSpmmProblem::run, spmvspmm.h:209). */
int daspmm_compat_spmm(int alg, int layout, int nr, int nc, int nnz, int nv,
                       const int *rowPtr, const int *rowIdx, const int *colIdx,
                       const float *values, const float *dnInput, float *dnOutput);

/* ---- Partition tables (bit-exact contract; used by tests) ----------------
 * Number of chunks for a nonzero-balanced split: max(1, ceil(nnz/chunk)). */
int daspmm_num_chunks(int nnz, int chunk);

/* Balanced-CSR boundaries on the device: meta[2c] = first nonzero of chunk c
 * after snapping, meta[2c+1] = its row; nchunks+1 entries (int pairs).
 * No reference counterpart (helper.h:283-321 has only a commented-out
 * binary_search_segment_number). */
daspmm_status daspmm_partition(int nr, int nnz, const int *rowPtr, int chunk,
                               int snap, int *meta, void *stream);

/* Output-row ownership the kernels realise: for each row r, owner[2r] = chunk
 * that writes it (or -1), owner[2r+1] = number of chunks holding a piece of
 * it.  alg = DASPMM_ALG_CSR_BALANCED (uses rowPtr) or DASPMM_ALG_COO_SCALAR
 * (uses rowIdx).  owner is device memory of 2*nr ints.  Runs the kernels'
 * own traversal with the arithmetic switched off. */
daspmm_status daspmm_ownership(int alg, int nr, int nnz, const int *rowPtr,
                               const int *rowIdx, int chunk, int snap, int *owner,
                               void *stream);

/* ---- Format conversion -----------------------------------------------------
 * Device COO -> CSR row pointer from sorted rowIdx[nnz]; rowPtr has nr+1
 * entries.  Bit-exact with generateCsrRowPtrArray
 * (spmvspmm_benchmark.cu:41-76), and defined for nnz == 0. */
daspmm_status daspmm_coo_to_csr(int nr, int nnz, const int *rowIdx, int *rowPtr,
                                void *stream);

/* ---- Mixed precision ---------------------------------------------------
 * C (FP32, row-major) = A*B + beta*C with A's values stored as val_fmt and B
 * as b_fmt; products and sums in FP32.  Supported (val_fmt, b_fmt):
 * (F32,F32), (BF16,BF16), (F16,F16), (F32,E4M3), (BF16,E4M3).  For E4M3, B
 * holds q with B[i,k] ~ q[i,k] * b_scales[k] (FP32 per-column scales, e.g.
 * from daspmm_e4m3_scales).  kahan_min > 0: rows with at least that many
 * nonzeros are summed with Kahan compensation.  Balanced-CSR split, row-major,
 * nv a multiple of 32; B aligned to its vector access (8 bytes for 16-bit,
 * 4 for FP8 at nv % 128 == 0).  workspace NULL: the library's per-stream one.
 * Extends the reference's FP32-only kernels (spmm.h:17-18: values and B are
 * float). */
daspmm_status daspmm_spmm_mixed(const daspmm_config *cfg, int layout, int nr, int nc,
                                int nnz, int nv, const int *rowPtr, const int *colIdx,
                                const void *values, int val_fmt, const void *B, int b_fmt,
                                const float *b_scales, float *C, float beta, int kahan_min,
                                void *workspace, size_t ws_bytes, void *stream);

/* q[i] = round_to_nearest_even(x[i] / col_scales[i % ncols]) in fmt (BF16,
 * F16, or E4M3 saturating to +-448); col_scales may be NULL (no division). */
daspmm_status daspmm_quantize(int fmt, size_t n, const float *x, void *q,
                              const float *col_scales, int ncols, void *stream);

/* Per-column E4M3 scales of a row-major nrows x ncols FP32 matrix:
 * scales[k] = max_i |B[i,k]| / 448 (1 for an all-zero column). */
daspmm_status daspmm_e4m3_scales(int nrows, int ncols, const float *B, float *scales,
                                 void *stream);

/* ---- Batched SpMM (one persistent launch for many problems) --------------
 * No counterpart in the reference (one problem per cudaSpmm call,
 * spmvspmm.h:53-199).  Every instance is C = A*B + beta*C with its own CSR A
 * (nr x nc, nnz), row-major B (nc x nv) and C (nr x nv); nv may differ
 * between instances (column tiles of 128, 64 or 32 by each instance's own nv),
 * the storage formats are the batch's (values F32 or BF16; B F32, BF16 or
 * E4M3 with b_scales).  How a row is summed depends only on its own matrix,
 * nv and chunk: a result is bit-identical whatever else is in the batch.  The device pointers must stay valid while the batch is used. */
typedef struct daspmm_instance {
    int nr, nc, nnz, nv;
    const int *rowPtr;
    const int *colIdx;
    const void *values;
    int val_fmt;
    const void *B;
    int b_fmt;
    const float *b_scales;
    float *C;
    float beta;
} daspmm_instance;

typedef struct daspmm_batch_s *daspmm_batch;

/* Cuts every matrix into tiles of about cfg->chunk nonzeros (default 256;
 * runs of whole rows, and rows longer than chunk cut into pieces of chunk
 * nonzeros whose partial sums are added in piece order by the row's last
 * piece), reading each rowPtr once on the host, and lists the work items
 * (instance, tile, column tile) on the device; synchronises `stream`.
 * DASPMM_ERR_BAD_MATRIX when a rowPtr is not a valid row pointer.  The batch
 * keeps scratch for the pieces: one batch must not run on two streams at
 * once.  cfg may be NULL. */
daspmm_status daspmm_batch_create(const daspmm_instance *inst, int n, const daspmm_config *cfg,
                                  daspmm_batch *out, void *stream);
/* One queue reset (memset) and one persistent kernel launch on `stream`. */
daspmm_status daspmm_batch_run(daspmm_batch b, void *stream);
/* Captures daspmm_batch_run on `stream` (not the legacy stream) into a CUDA
 * graph kept in the batch; daspmm_batch_replay launches it. */
daspmm_status daspmm_batch_capture(daspmm_batch b, void *stream);
daspmm_status daspmm_batch_replay(daspmm_batch b, void *stream);
daspmm_status daspmm_batch_info(daspmm_batch b, long long *nitems, long long *total_nnz);
daspmm_status daspmm_batch_destroy(daspmm_batch b);
/* Autotunes the batch's row-tile size: times daspmm_batch_run for each
 * chunk in chunks[0..nchunks) (NULL: 128, 256, 512, 1024), reps runs each,
 * and returns the fastest (C of every instance is overwritten). */
daspmm_status daspmm_batch_tune(const daspmm_instance *inst, int n, const int *chunks,
                                int nchunks, int reps, int *best_chunk, float *best_us,
                                void *stream);
/* No counterpart in the reference.  Tunes the row-tile size and the column-
 * tile width together: for every width in `widths` (floats: 128, 64 or 32;
 * NULL = all three; an instance's tile is the widest of 128 / 64 / 32 that
 * divides its nv and is at most the width) the fastest of `chunks` (NULL =
 * 128, 256, 512, 1024), each batch timed over `reps` runs.  *best receives
 * the winning daspmm_batch_create config (chunk, lanes_col = width / 4).
 * Results do not depend on either choice. */
daspmm_status daspmm_batch_tune_ex(const daspmm_instance *inst, int n, const int *chunks,
                                   int nchunks, const int *widths, int nwidths, int reps,
                                   daspmm_config *best, float *best_us, void *stream);

/* ---- Matrix Market input ---------------------------------------------------
 * Coordinate files (real, integer or pattern values; general, symmetric,
 * skew-symmetric or hermitian) to CSR sorted by (row, col).  Replaces
 * readMtx (util/spmatrix.hpp:286-333) with makeSymmetric
 * (spmatrix.hpp:219-284): a symmetric file is mirrored and loses its diagonal
 * and repeated (row, col) pairs, as in the reference, but every value stays
 * with its own (row, col) (the reference compacts rows and columns only, so
 * its values after the first dropped entry are misplaced).  Skew-symmetric
 * and hermitian files are read as stored (the reference does not mirror
 * them either); pattern entries have value 1; repeated pairs of a general
 * file are kept, in file order. */
#define DASPMM_MTX_KEEP_DIAGONAL 1   /* symmetric files: keep diagonal entries */

typedef struct daspmm_mtx_header {
    int nr, nc;
    long long entries;   /* entries stored in the file */
    int field;           /* 0 real, 1 integer, 2 pattern, 3 complex */
    int symmetry;        /* 0 general, 1 symmetric, 2 skew-symmetric, 3 hermitian */
    long long nnz_max;   /* capacity that daspmm_mtx_read needs at most */
} daspmm_mtx_header;

daspmm_status daspmm_mtx_info(const char *path, daspmm_mtx_header *out);
/* Host arrays: rowPtr[nr+1]; rowIdx (may be NULL: the COO row of each
 * nonzero), colIdx and values of capacity `cap` (>= the nonzeros produced,
 * DASPMM_ERR_WORKSPACE otherwise).  DASPMM_ERR_BAD_MATRIX for a malformed
 * file (bad banner or size line, an index out of range, fewer entries than
 * the size line says); DASPMM_ERR_UNSUPPORTED for complex or dense files. */
daspmm_status daspmm_mtx_read(const char *path, int flags, long long cap, int *rowPtr,
                              int *rowIdx, int *colIdx, float *values, int *nnz_out);

/* ---- CSR validation -------------------------------------------------------
 * Checks a device CSR matrix: rowPtr[0] == 0, rowPtr[nr] == nnz, rowPtr
 * non-decreasing, every colIdx in [0, nc) and, with sorted != 0, strictly
 * increasing columns inside each row (the driver's order, spmatrix.hpp:327).
 * Synchronises `stream`.  DASPMM_ERR_BAD_MATRIX with *bad_row = the first
 * offending row (when bad_row is not NULL; -1 otherwise).  The reference
 * checks nothing (spmvspmm_benchmark.cu:41-76 trusts a sorted rowIdx). */
daspmm_status daspmm_csr_check(int nr, int nc, int nnz, const int *rowPtr, const int *colIdx,
                               int sorted, int *bad_row, void *stream);

/* ---- Serving loop ----------------------------------------------------------
 * No counterpart in the reference (SpmvSpmmProblem::benchmark times one
 * problem in a loop, spmvspmm.h:220-243).  A server owns a CUDA stream on
 * the device current at creation, a pool of device-resident CSR matrices
 * (caller-owned device arrays, checked once by daspmm_csr_check when added),
 * an output arena of budget_bytes device bytes and a dispatcher thread.
 * A request is C = A_m * B (FP32 C, row-major nr x nv, placed in the arena);
 * B is caller-owned device memory (row-major nc x nv in the server's b_fmt)
 * that must stay valid until the request finishes.
 *   admission: requests are launched in FIFO order once their C fits the
 *     arena; C stays allocated until daspmm_server_release.  A request whose
 *     C alone exceeds the budget is refused at submission (DASPMM_ERR_BUDGET).
 *   DASPMM_SERVE_BATCHED: each matrix is cut into tiles once when added (see
 *     daspmm_batch_create); whenever fewer than max_inflight launch groups are
 *     in flight, everything queued (up to max_batch requests and max_items
 *     work items) goes into one persistent batched launch (see daspmm_batch_*);
 *     with window_us > 0 and the GPU busy, a group is held back until its
 *     oldest request has waited window_us or max_batch requests are queued.
 *     A request's result does not depend on which group it lands in.
 *   DASPMM_SERVE_PLAIN: one daspmm_spmm (balanced CSR, FP32) launch per
 *     request; val_fmt and b_fmt must be DASPMM_F32.
 * Latency: from arrival (submission, or the scheduled time in
 * daspmm_server_replay) to the dispatcher seeing the launch's event. */
#define DASPMM_SERVE_BATCHED 0
#define DASPMM_SERVE_PLAIN 1

typedef struct daspmm_server_config {
    long long budget_bytes;  /* output arena bytes; 0: 1 GiB */
    int mode;                /* DASPMM_SERVE_BATCHED or DASPMM_SERVE_PLAIN */
    int val_fmt, b_fmt;      /* storage of every matrix's values / every B */
    int chunk;               /* batched: nonzeros per row tile; 0: 256 */
    int max_batch;           /* batched: requests per launch; 0: 1024 */
    int max_inflight;        /* launch groups in flight; 0: 2 batched, 64 plain */
    int window_us;           /* batched: batching window while the GPU is busy */
    long long max_items;     /* batched: work items per launch; 0: 1 << 22 */
    long long scratch_bytes; /* batched: row-piece sums per launch group; 0: 64 MiB */
} daspmm_server_config;

typedef struct daspmm_request {
    int matrix;              /* id from daspmm_server_add_matrix */
    int nv;
    const void *B;
    const float *b_scales;   /* E4M3 B: per-column scales */
} daspmm_request;

typedef struct daspmm_result {
    int status;              /* DASPMM_OK, DASPMM_ERR_CANCELLED, ...; -1 pending */
    int group;               /* launch group that served it (-1: none) */
    float *C;                /* device result in the arena until released */
    double queue_us;         /* arrival -> launch */
    double latency_us;       /* arrival -> completion seen */
} daspmm_result;

typedef struct daspmm_serve_stats {
    long long completed, cancelled, refused, groups, launched, items, queued;
    long long arena_used, arena_bytes;
    int max_group, inflight_groups, matrices, error;
} daspmm_serve_stats;

typedef struct daspmm_server_s *daspmm_server;

daspmm_status daspmm_server_create(const daspmm_server_config *cfg, daspmm_server *out);
/* Adds a resident matrix (device rowPtr/colIdx/values, complete before the
 * call); DASPMM_ERR_BAD_MATRIX when it fails the CSR check. */
daspmm_status daspmm_server_add_matrix(daspmm_server s, int nr, int nc, int nnz,
                                       const int *rowPtr, const int *colIdx,
                                       const void *values, int *id);
daspmm_status daspmm_server_submit(daspmm_server s, const daspmm_request *r, long long *ticket);
/* Removes a request that is still queued (DASPMM_ERR_UNSUPPORTED once it
 * has been launched); its result reports DASPMM_ERR_CANCELLED. */
daspmm_status daspmm_server_cancel(daspmm_server s, long long ticket);
/* Waits for a request (timeout_ms < 0: no limit; DASPMM_ERR_TIMEOUT when it
 * expires).  The result stays readable until daspmm_server_release. */
daspmm_status daspmm_server_wait(daspmm_server s, long long ticket, int timeout_ms,
                                 daspmm_result *out);
/* Frees a finished request's C and forgets it. */
daspmm_status daspmm_server_release(daspmm_server s, long long ticket);
/* Open-loop load from the calling thread: submits reqs[i] at arrival_s[i]
 * seconds after the call, waits for all and fills results[i] (refused
 * submissions carry their status).  release != 0 frees every C at once. */
daspmm_status daspmm_server_replay(daspmm_server s, const daspmm_request *reqs, int n,
                                   const double *arrival_s, int release,
                                   daspmm_result *results);
daspmm_status daspmm_server_stats(daspmm_server s, daspmm_serve_stats *out);
/* Cancels queued requests, lets launched ones finish, frees everything. */
daspmm_status daspmm_server_destroy(daspmm_server s);

/* ---- Host buffers ------------------------------------------------------
 * The same product with A, B and C in HOST memory (pinned or pageable): the
 * library copies A and B to device buffers it keeps per (device, stream),
 * runs daspmm_spmm_ex, copies C back and synchronises the stream before it
 * returns.  C is read (copied in) only when beta != 0.  rowIdx may be NULL
 * for CSR algorithms and rowPtr NULL for COO algorithms.  The entry point
 * of a caller that holds its matrices on the host (the reference's driver
 * copies them itself, spmvspmm_benchmark.cu:369-383). */
daspmm_status daspmm_spmm_host(const daspmm_config *cfg, int layout, int nr, int nc,
                               int nnz, int nv, const int *rowPtr, const int *rowIdx,
                               const int *colIdx, const float *values, const float *B,
                               float *C, float beta, void *stream);
/* daspmm_spmm_host without the final synchronisation: the copies and the
 * SpMM are queued on `stream` and the call returns.  A, B and C (host) must
 * stay untouched until the stream has finished.  Calls on one stream share
 * that stream's device staging (stream order keeps them apart); calls on
 * different streams overlap one another's copies in both directions. */
daspmm_status daspmm_spmm_host_async(const daspmm_config *cfg, int layout, int nr, int nc,
                                     int nnz, int nv, const int *rowPtr, const int *rowIdx,
                                     const int *colIdx, const float *values, const float *B,
                                     float *C, float beta, void *stream);

/* ---- Planned SpMM: one matrix, many products ---------------------------
 * No counterpart in the reference (its benchmark loop, spmvspmm.h:220-243,
 * times one problem; its kernels need no partition).  daspmm_spmm recomputes
 * the balanced split's chunk boundaries (a pass over rowPtr) in every call,
 * so the matrix may change between calls.  A plan fixes the matrix (device
 * rowPtr / colIdx / values, which must stay unchanged and alive until
 * daspmm_plan_destroy), row-major layout and nv: the boundaries are computed
 * once, into a workspace the plan owns, and each daspmm_plan_spmm with beta
 * == 0 and B / C 32-byte aligned is one launch of the window kernel.  Results
 * are bit-identical to daspmm_spmm with the plan's configuration.  Other calls
 * (beta != 0, other alignment) take the stateless path on the plan's
 * workspace.  cfg: NULL or {.alg = DASPMM_ALG_CSR_BALANCED, ...}.
 * daspmm_plan_create allocates (cudaMalloc) and synchronises `stream`.
 * Calls on one plan share its workspace: order them (one stream); calls that
 * overlap on the GPU race. */
typedef struct daspmm_plan_s *daspmm_plan;
daspmm_status daspmm_plan_create(const daspmm_config *cfg, int nr, int nc, int nnz, int nv,
                                 const int *rowPtr, const int *colIdx, const float *values,
                                 void *stream, daspmm_plan *out);
daspmm_status daspmm_plan_spmm(daspmm_plan p, const float *B, float *C, float beta,
                               void *stream);
daspmm_status daspmm_plan_config(daspmm_plan p, daspmm_config *out);
daspmm_status daspmm_plan_destroy(daspmm_plan p);

/* ---- No device allocation ----------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * -- a plugin inside an application whose own allocator owns the device's
 * memory, or a loop that must not pay the device-wide synchronisation of
 * cudaMalloc/cudaFree.  Same product as daspmm_spmm with
 * DASPMM_ALG_CSR_BALANCED on the same inputs and outputs (C = A*B + beta*C,
 * row- or col-major), but the scratch it needs lives in a fixed array of
 * DASPMM_NOALLOC_MAX_BYTES inside the library, which every GPU that loads the
 * library keeps until the process exits.  Nothing is allocated, by this
 * library or any other.
 *   - Limit: daspmm_workspace_bytes(cfg, layout, nr, nc, nnz, nv) must be
 *     <= DASPMM_NOALLOC_MAX_BYTES, with cfg = {.alg = DASPMM_ALG_CSR_BALANCED}
 *     for row-major and {.alg = DASPMM_ALG_CSR_BALANCED, .pipe = 1} for
 *     column-major (this entry point gathers column-major B directly, since
 *     the transposing path would need room for copies of B and C).  That is
 *     about 8 * nchunks * nv bytes (two carry rows per chunk), with nchunks =
 *     ceil(nnz / chunk): row-major chunk = 96 for nv = 128, 64 for nv = 64
 *     and 128 for the other nv that are multiples of 32 (32..128 otherwise);
 *     column-major chunk = 32.  So row-major nv = 128 fits up to about 1.6 M
 *     nonzeros (the 262,144-row power-law matrix, 1.24 M, needs 13.4 MB),
 *     nv = 32 about 8 M; column-major nv = 16 about 4 M.  Larger problems
 *     return DASPMM_ERR_WORKSPACE before any device work.
 *   - The first call on each device (and the first after a cudaDeviceReset
 *     of it) looks up the array's device address with that device current;
 *     make that call before any stream capture.
 *   - All calls on a device share the one array.  Calls that overlap on the
 *     GPU (different streams, or different host threads, without ordering
 *     between them) race on it; order them.  The array keeps the last call's
 *     contents; each call writes every entry it reads, so none needs
 *     clearing. */
#define DASPMM_NOALLOC_MAX_BYTES (16u << 20)
daspmm_status daspmm_spmm_noalloc(int layout, int nr, int nc, int nnz, int nv,
                                  const int *rowPtr, const int *colIdx,
                                  const float *values, const float *B, float *C,
                                  float beta, void *stream);

/* ---- L2 persistence ---------------------------------------------------
 * No counterpart in the reference.  Sets the current device's persisting L2
 * set-aside (cudaLimitPersistingL2CacheSize) for this process's context, used
 * by launches whose config has l2_window > 0, at most the device's largest
 * (cudaDevAttrMaxPersistingL2CacheSize; larger requests are clamped to it);
 * 0 resets it and returns the persisting lines to normal
 * (cudaCtxResetPersistingL2Cache).  The setting is
 * the context's: it ends with the process and applies to all of its work on
 * the device. */
daspmm_status daspmm_l2_set_aside(size_t bytes);

/* ---- Diagnostics ------------------------------------------------------- */
/* Reads and clears the device-side error word of the current device: 0, or
 * DASPMM_ERR_TIMEOUT if a kernel's bounded wait expired since the last call
 * (that kernel stopped early and its output is incomplete). */
daspmm_status daspmm_device_error(void);

/* No counterpart in the reference.  Runs the bounded shared-memory barrier
 * wait the ring kernels (pipes 2 and 3) use, alone, in one thread of one CTA:
 * with `expire` != 0 the barrier expects bytes that nothing delivers (no copy
 * is issued), so the wait gives up after `polls` polls, sets the device error
 * word (read by daspmm_device_error) and the kernel returns; with expire == 0
 * the wait succeeds at once.  Writes out[0] (device int) = 1 when the wait
 * succeeded, 0 when it expired.  Asynchronous on `stream`. */
daspmm_status daspmm_wait_probe(int polls, int expire, int *out, void *stream);

/* Number of kernels this library has launched in this process. */
long long daspmm_launch_count(void);

/* Kernel timing for benchmarks.  After daspmm_kernel_timer_begin(n), each
 * SpMM call (of any thread, on the current device) records a pair of CUDA
 * events, created by the library, immediately before and after the launch of
 * its main gather kernel on the call's stream; slots 0..n-1 are used once
 * each, later calls are not timed.  daspmm_kernel_timer_end waits for the
 * recorded events, writes up to n elapsed times (ms) to ms_out, releases the
 * events and returns how many calls were timed (or -1 on a CUDA error). */
daspmm_status daspmm_kernel_timer_begin(int n);
int daspmm_kernel_timer_end(float *ms_out, int n);

const char *daspmm_status_string(daspmm_status s);
int daspmm_last_cuda_error(void);   /* cudaError_t of the last failure on this thread */
int daspmm_abi_version(void);

/* ---- Host-side synthetic inputs (deterministic for a seed) -----------------
 * Exactly `per_row` distinct uniformly random columns per row, sorted; values
 * U(-1,1).  rowPtr[nr+1], colIdx/values[nr*per_row]. */
daspmm_status daspmm_gen_uniform(int nr, int nc, int per_row, uint64_t seed,
                                 int *rowPtr, int *colIdx, float *values);

/* Power-law graph: out-degree k in [dmin, dmax] with p(k) ~ (k + shift)^-alpha,
 * columns by preferential attachment (probability ~ in-degree + 1, duplicates
 * in a row redrawn), values U(-1,1).  Two calls: first with colIdx == NULL to
 * get rowPtr (returns nnz in *nnz_out), then with the arrays allocated.
 * mean_scale != 1 multiplies every degree (rounded, clamped to [dmin, dmax]),
 * for families with a target average degree. */
daspmm_status daspmm_gen_powerlaw(int nr, int nc, double alpha, double shift,
                                  int dmin, int dmax, double mean_scale,
                                  uint64_t seed, int *rowPtr, int *colIdx,
                                  float *values, long long *nnz_out);

/* Uniform random sparse matrix with Poisson(avg_deg) distinct columns per row
 * (two calls as above). */
daspmm_status daspmm_gen_random(int nr, int nc, double avg_deg, uint64_t seed,
                                int *rowPtr, int *colIdx, float *values,
                                long long *nnz_out);

/* n floats U(lo, hi). */
void daspmm_gen_dense(size_t n, uint64_t seed, float lo, float hi, float *out);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* DASPMM_H */
