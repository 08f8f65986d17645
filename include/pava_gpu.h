/*
 * pava_gpu.h -- C ABI of the pava B200 SpMV engine (sm_100a).
 *
 * Plain pointers, sizes and status codes only; device pointers are CUDA device addresses and
 * a stream is passed as `void *` (a cudaStream_t, or NULL for the default stream).  Every entry
 * point returns a pava_status (or the reference's int convention where it mirrors a
 * reference function), never exits and never aborts.
 *
 * Each declaration names the reference interface it replaces (path:line in the reference
 * tree).  The engine is CUDA throughout: there is no CPU fallback, and an entry point that
 * needs the GPU reports PAVA_E_CUDA when none is usable.
 */
#ifndef PAVA_GPU_H
#define PAVA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  0 .. -5 keep the values of the reference's ANONYMOUSLIB codes
 * (csr5/detail/common.h:13-18); the rest are new. */
typedef enum pava_status {
    PAVA_SUCCESS = 0,                  /* ANONYMOUSLIB_SUCCESS */
    PAVA_E_UNKNOWN_FORMAT = -1,        /* ANONYMOUSLIB_UNKOWN_FORMAT */
    PAVA_E_UNSUPPORTED_PARAMS = -2,    /* ANONYMOUSLIB_UNSUPPORTED_CSR5_OMEGA: tile parameters */
    PAVA_E_CONVERT_FAILED = -3,        /* ANONYMOUSLIB_CSR_TO_CSR5_FAILED */
    PAVA_E_NOT_CONVERTED = -4,         /* ANONYMOUSLIB_UNSUPPORTED_CSR_SPMV: spmv before asCSR5 */
    PAVA_E_UNSUPPORTED_VALUE_TYPE = -5,/* ANONYMOUSLIB_UNSUPPORTED_VALUE_TYPE */
    PAVA_E_INVALID_ARG = -10,
    PAVA_E_INVALID_CSR = -11,          /* row_ptr not monotone / column out of range */
    PAVA_E_CUDA = -12,                 /* CUDA error or no usable GPU */
    PAVA_E_NOMEM = -13,
    PAVA_E_TIMEOUT = -14,              /* a bounded device wait gave up */
    PAVA_E_TOO_LARGE = -15             /* sizes beyond the int32 element space */
} pava_status;

/* Storage formats.  CSR and CSR5 keep the reference's ANONYMOUSLIB_FORMAT_* values
 * (csr5/detail/common.h:20-22); CVR is cvr/cvr.h's format. */
typedef enum pava_format {
    PAVA_FORMAT_CSR = 0,   /* plain CSR, row-group kernel (lanes per row, SpMM, batches) */
    PAVA_FORMAT_CSR5 = 1,  /* CSR5 tiles: 32 lanes x sigma, bit-flag descriptors */
    PAVA_FORMAT_CVR = 3,   /* CVR chunks: 32 lanes x S steps, row-completion bits */
    PAVA_FORMAT_SELL = 4   /* sliced ELLPACK: slices of 32 rows, one lane per row, rows padded
                              to the slice's longest (rounded up to 4); refused
                              (PAVA_E_UNSUPPORTED_PARAMS) when padding would more than double
                              the stored elements.  No counterpart in the reference. */
} pava_format;

typedef enum pava_precision {
    PAVA_PREC_FP64 = 0,    /* values, x, y FP64; FMA accumulation */
    PAVA_PREC_FP32C = 1    /* values and x FP32, FP64 y.  CVR / CSR5: compensated FP32
                              accumulation, FP64 carries; SELL: the exact FP32 products
                              summed in FP64 */
} pava_precision;

typedef enum pava_index_mode {
    PAVA_INDEX_I32 = 0,     /* 32-bit column indices */
    PAVA_INDEX_DELTA16 = 1, /* 16-bit column offsets from a per-chunk base column, the middle
                               of the chunk's column range (every chunk's columns within a
                               span of 65534, else PAVA_E_UNSUPPORTED_PARAMS) */
    PAVA_INDEX_AUTO = 2     /* CVR / CSR5: 16-bit offsets when every column fits, otherwise
                               32-bit columns (pava_info.index_mode tells which); same results */
} pava_index_mode;

/* A CSR matrix, 0-based, sorted or unsorted columns, FP64 values (the reference's
 * _PAVA_CSRMatrix, utils/basicMatrix.h:51-60). */
typedef struct pava_csr {
    int m, n, nnz;
    const int *row_ptr;   /* m + 1 */
    const int *col_idx;   /* nnz   */
    const double *vals;   /* nnz   */
    int on_device;        /* 1: the three arrays are device memory; 0: host memory */
} pava_csr;

/* Tuning knobs; zero means "default". */
typedef struct pava_opts {
    int steps;            /* CVR: steps per warp chunk, 32, 64 or 128 (default 64; 32 when a
                             matrix gives fewer than 24 chunks of 64 steps per SM) */
    int sigma;            /* CSR5: elements per lane per tile, 8, 12, 16, 24 or 32 (default 16) */
    int tiles_per_chunk;  /* CSR5: tiles per warp chunk, 1 .. 64 (default 4; 2 or 1 when a
                             matrix gives fewer than 4 x 24 tiles per SM), or PAVA_TILES_WAVE
                             (-1): the count in 1 .. 8 that fills the last wave of resident
                             warps best for this matrix */
    int precision;        /* pava_precision */
    int index_mode;       /* pava_index_mode */
    int lanes_per_row;    /* CSR: lanes per row group, 1, 2, 4, 8, 16 or 32 (default: from
                             the mean row length, or from k for pava_spmm); SELL: lanes per
                             row of pava_spmm, 4, 8 or 16 (default: from k) */
    int col_lanes;        /* CSR, pava_spmm: lanes of a group across the k right-hand sides,
                             a power of two <= lanes_per_row (default: from k) */
    int cols_per_lane;    /* CSR, pava_spmm: right-hand sides per lane, 1, 2 or 4; needs
                             col_lanes * cols_per_lane >= k (default: from k) */
    int rows_per_tile;    /* CSR: rows per warp tile of the persistent launch, a multiple of
                             32 / lanes_per_row (default: 4 row groups); with x_window, rows
                             per 256-thread CTA tile, a multiple of 8 * 32 / lanes_per_row
                             (default: 4 passes of the CTA's row groups) */
    int x_window;         /* CSR, pava_spmm: 1 = each CTA copies its row tile's column window
                             of X into shared memory (up to 100 KB) and reads X from there;
                             for banded / local matrices.  Tiles whose window is wider read X
                             from global memory. */
} pava_opts;

typedef struct pava_info {
    int format, precision, index_mode;
    int m, n, nnz, n_empty;
    long long chunks;          /* warp chunks (CVR, CSR5) or rows (CSR) */
    long long elems_per_chunk;
    double convert_ms;         /* device time of the conversion */
    size_t device_bytes;       /* bytes the handle holds on the device */
    double alg_bytes;          /* compulsory bytes of one SpMV: nnz*(s_v+s_i) + 4(m+1) + n*s_x
                                  + m*s_y (x and y counted once) */
    double format_bytes;       /* bytes one SpMV streams from the format (values, columns,
                                  flags, metadata) plus x and y */
} pava_info;

typedef struct pava_handle pava_handle;

/* Selects the CUDA device for the calling thread (cudaSetDevice). */
pava_status pava_init(int device);

/* Device memory budget of one handle (process-wide setting; 0, the default, means none): a
 * pava_create whose format arrays would take more than `bytes` fails with PAVA_E_NOMEM and
 * frees what it allocated, as when the device itself runs out.  The reference sizes nothing
 * (its arrays are _mm_malloc'd unchecked, cvr/cvr.h:2008-2030).  No GPU needed to set it. */
pava_status pava_set_device_memory_limit(unsigned long long bytes);
unsigned long long pava_get_device_memory_limit(void);

/* Bounds-checked builds (python -m pava_b200.build --bounds: libpava_gpu_bounds.so, compiled
 * with PAVA_BOUNDS_CHECK).  Their SpMV kernels test every index that comes from data -- each
 * x gather's column, each y row, slot numbers and tail counts read from the format's metadata,
 * the carry chunk of a shared row -- and skip an access that would leave its array, counting
 * it instead of faulting.  pava_bounds_checked() says whether this library is such a build;
 * pava_bounds_report(out3, clear) synchronises the device and returns the count of failed
 * tests, the site of the first (1 x, 2 y, 3 carry, 4 shared slot) and its index, clearing them
 * when `clear` is set (PAVA_E_UNSUPPORTED_PARAMS in ordinary builds).  The reference has no
 * checked build (it reads and writes its arrays unchecked); this stands in for a memory
 * checker where none may run. */
int pava_bounds_checked(void);
pava_status pava_bounds_report(unsigned long long *out3, int clear);

/* Bounded waits.  The SELL SpMV waits on mbarriers for its bulk copies into shared memory;
 * each wait gives up after about a second, counts itself in a device word and lets the kernel
 * finish instead of hanging.  pava_wait_report(out2, clear) synchronises the device and
 * returns PAVA_E_TIMEOUT when a wait gave up since the last clear (PAVA_SUCCESS otherwise),
 * with out2 = {waits that gave up, the first one's slice + 1}; `clear` resets the word.  No
 * reference counterpart (the reference's CPU code never waits on the device). */
pava_status pava_wait_report(unsigned long long *out2, int clear);

/* Converts A into `format` on the device (the GPU form of anonymouslibHandle::inputCSR +
 * asCSR5, csr5/anonymouslib_avx512.h:58-70,107-221, and of CVR's pre_processing,
 * cvr/cvr.h:583-1060).  The caller's arrays are never modified (the reference transposes
 * them in place, format_avx512.h:428).  The conversion is validated first: a row_ptr that
 * is not monotone or a column outside [0, n) gives PAVA_E_INVALID_CSR.  Sizes: the CVR and
 * CSR5 forms index their padded element space with int32, so nnz + 65,600 >= 2^31 (checked
 * before any array is read) or a padded space past 2^31 - 64 gives PAVA_E_TOO_LARGE, as does
 * m = 2^31 - 1; a device allocation that fails, or that passes the memory budget of
 * pava_set_device_memory_limit, gives PAVA_E_NOMEM with nothing left allocated. */
pava_status pava_create(const pava_csr *A, int format, const pava_opts *opts, void *stream,
                        pava_handle **out);

/* y = A x on the device (anonymouslibHandle::spmv, csr5/anonymouslib_avx512.h:234-256;
 * spmv_compute_kernel, cvr/cvr.h:1062).  FP64 handles take double x and write double y;
 * FP32C handles take float x and write double y.  Every call overwrites all m entries of y
 * (empty rows become 0), so repeated calls give identical results -- unlike the reference,
 * whose repeated calls accumulate into shared rows (cvr/cvr.h:1415; csr5_spmv_avx512.h:277). */
pava_status pava_spmv(pava_handle *h, const void *x, void *y, void *stream);

/* Y = A X for k right-hand sides: X is n x k and Y is m x k, both row-major with leading
 * dimensions ldx >= k and ldy >= k (elements), device memory; FP64, or FP32C with float X and
 * double Y.  CSR handles (the row-group kernel), 1 <= k <= 128, and SELL handles (a CTA per
 * 32-row slice, the slice's streams in shared memory, opts.lanes_per_row = 4, 8 or 16 lanes
 * per row across k; 0 = 4 for k <= 16, else 8), 1 <= k <= 64, k <= 32 with 4 lanes
 * (PAVA_E_UNSUPPORTED_PARAMS past it).  The reference has no multi-vector product; k = 1
 * equals pava_spmv. */
pava_status pava_spmm(pava_handle *h, int k, const void *X, long long ldx, void *Y,
                      long long ldy, void *stream);
/* pava_spmv split into its launches, for timing one kernel: stage 1 runs the format's SpMV
 * kernel, stage 2 the carry fixup that finishes rows shared between warp chunks (CVR and
 * CSR5; a no-op for CSR), stage 0 both (= pava_spmv).  y is complete only after stage 2.
 * No counterpart in the reference. */
pava_status pava_spmv_stage(pava_handle *h, const void *x, void *y, void *stream, int stage);

/* End-to-end form of pava_spmv on host buffers: copies x host->device, runs the SpMV and
 * copies y device->host on `stream`, then synchronises it.  Buffers for x and y are kept on
 * the handle after the first call. */
pava_status pava_spmv_host(pava_handle *h, const void *x_host, void *y_host, void *stream);

/* Pipelined form of pava_spmv_host: queues the copy of x in, the SpMV and the copy of y out on
 * the handle's own streams and returns at once, so that consecutive calls overlap one call's
 * copy-in, another's SpMV and a third's copy-out (two staging slots).  `stream` waits for the
 * call's copy-out.  The copy-in does not wait for `stream`: x_host must hold its values when
 * the call is made.  x_host and y_host should be pinned, and must stay untouched until the call
 * is complete: after pava_spmv_host_wait, or once `stream` has reached the point of the call.
 * No counterpart in the reference. */
pava_status pava_spmv_host_async(pava_handle *h, const void *x_host, void *y_host,
                                 void *stream);
/* Waits until every pava_spmv_host_async call on the handle is complete. */
pava_status pava_spmv_host_wait(pava_handle *h);
pava_status pava_get_info(const pava_handle *h, pava_info *out);

/* anonymouslibHandle::destroy / asCSR (csr5/anonymouslib_avx512.h:80-104,258-262). */
pava_status pava_destroy(pava_handle *h);

/* Message of the last failed call on this thread ("" if none). */
const char *pava_last_error(void);
const char *pava_status_string(int status);

/* y = A x straight from a CSR already in device memory, allocating nothing: for callers that
 * may not call the CUDA allocator because a host framework owns the device memory and hands
 * them only pre-allocated buffers (or because their memory budget is already committed), and
 * so cannot create a handle.  No counterpart in the reference.
 *   - Scratch: a 1 MiB array compiled into this library (held on every GPU that loads it until
 *     the process exits), enough for 32,768 chunks of 4,096 nonzeros: nnz above 134,217,728
 *     returns PAVA_E_TOO_LARGE and launches nothing.
 *   - The first call on a device looks up the array's device address on the current device
 *     (cudaGetSymbolAddress); make that first call before any stream capture.  The address is
 *     kept for the life of the process: cudaDeviceReset on that device makes it stale, so a
 *     process that resets the device must not call this entry point on it again.
 *   - All calls share the array: calls that overlap on the GPU (other streams, other threads)
 *     race and must be serialised by the caller.  Each call rewrites every slot it reads.
 *   - The CSR must be valid (non-decreasing row_ptr, row_ptr[m] == nnz, columns in [0, n)); it
 *     is not checked.  Empty rows get y = 0; results agree with pava_spmv within rounding. */
pava_status pava_spmv_csr_noalloc(int m, int n, int nnz, const int *row_ptr, const int *col_idx,
                                  const double *vals, const double *x, double *y, void *stream);

/* ---- Batches of independent matrices ------------------------------------------------
 * No counterpart in the reference (its benchmark loop runs one matrix at a time,
 * main.cpp:554-587).  A batch holds the block-diagonal union of `count` matrices: x and y
 * of the batch are the matrices' x and y concatenated (offsets from pava_batch_layout), so
 * one SpMV over the union -- one launch, persistent for the CSR form -- serves all of them. */
typedef struct pava_batch pava_batch;
/* mats[i] is a CSR (host or device arrays per its on_device flag), validated per matrix.
 * format < 0 autotunes the union over the built-in candidates (pava_autotune, k = 1) and
 * keeps the fastest; otherwise format/opts are used as in pava_create.  Sums of rows,
 * columns and nonzeros must stay below 2^31 (PAVA_E_TOO_LARGE). */
pava_status pava_batch_create(int count, const pava_csr *mats, int format,
                              const pava_opts *opts, void *stream, pava_batch **out);
/* The same for k right-hand sides per matrix (1 <= k <= 128): format < 0 autotunes the union
 * for k (pava_autotune over its candidates for k; for k > 1 the CSR row-group shapes), and a
 * given format must be PAVA_FORMAT_CSR when k > 1.  pava_batch_create is this with k = 1.
 * The reference's loop runs one matrix and one vector at a time (main.cpp:554-587). */
pava_status pava_batch_create_spmm(int count, const pava_csr *mats, int k, int format,
                                   const pava_opts *opts, void *stream, pava_batch **out);
/* count + 1 prefix offsets of each matrix's x, y and nonzeros in the union (any may be NULL). */
pava_status pava_batch_layout(const pava_batch *b, long long *x_offsets, long long *y_offsets,
                              long long *nnz_offsets);
/* The chosen form and the union's pava_info (any may be NULL). */
pava_status pava_batch_get(const pava_batch *b, int *format, pava_opts *opts, pava_info *info);
/* y = U x for the whole batch (x, y device buffers of the union's n and m). */
pava_status pava_batch_spmv(pava_batch *b, const void *x, void *y, void *stream);
/* Y = U X for the whole batch with k right-hand sides: X (union n x k) and Y (union m x k)
 * row-major with leading dimensions ldx, ldy >= k, matrix i's block at rows x_offsets[i] of X
 * and y_offsets[i] of Y; one persistent launch of the row-group SpMM (CSR-form batches, as
 * pava_spmm). */
pava_status pava_batch_spmm(pava_batch *b, int k, const void *X, long long ldx, void *Y,
                            long long ldy, void *stream);
/* Records the batch SpMV on (x, y) into a CUDA graph owned by the batch (replacing any
 * earlier one); pava_batch_replay launches it on `stream`. */
pava_status pava_batch_capture(pava_batch *b, const void *x, void *y);
/* Records the batch SpMM on (X, Y) into the batch's graph (replacing any earlier one). */
pava_status pava_batch_capture_spmm(pava_batch *b, int k, const void *X, long long ldx, void *Y,
                                    long long ldy);
pava_status pava_batch_replay(pava_batch *b, void *stream);
pava_status pava_batch_destroy(pava_batch *b);

/* ---- Exhaustive autotuner ------------------------------------------------------------
 * Converts A into every built-in candidate form for k right-hand sides and times each (two
 * warm-up calls, then the median of `reps` CUDA-event timings of the SpMV/SpMM with x and y
 * already on the device).  Candidates: for k = 1, CVR steps 64/128 and CSR5 sigma 16/32, each
 * with 32-bit columns and with PAVA_INDEX_AUTO (16-bit offsets where they reach), CSR5 also
 * with the tiles per chunk that fill the last wave of warp chunks best (1..8); for
 * every k, the CSR row-group form over lanes_per_row x col_lanes x cols_per_lane x
 * rows_per_tile, and for k > 1 also with x_window.  entries[0 .. *n_entries) receive every candidate (ms < 0 when it failed,
 * with its status), *best the index of the fastest.  No counterpart in the reference. */
typedef struct pava_tune_entry {
    int format;
    pava_opts opts;
    double ms;
    int status;
} pava_tune_entry;
pava_status pava_autotune(const pava_csr *A, int k, int precision, int reps,
                          pava_tune_entry *entries, int max_entries, int *n_entries, int *best);

/* ---- Device-side generators --------------------------------------------------------
 * Seeded synthetic matrices built on the GPU (one thread per row for the lengths, one per
 * nonzero for columns and values), for workloads too large to build on the host.  Columns
 * are sorted and distinct per row, values N(0,1).  No counterpart in the reference (it
 * reads .mtx files, utils/basicMatrix.cpp:63-253).  Families and parameters:
 *   STENCIL   p0 = dimensions (2 or 3), p1 = points (5/9 in 2-D, 7/27 in 3-D); m is rounded
 *             down to a g^d grid
 *   BANDED    p0 = half-bandwidth, p1 = nonzeros per row (clipped to the band)
 *   POWERLAW  p0 = mean row length, p1 = lognormal sigma, p2 = cap, p3 = share of empty rows
 *   BLOCKDIAG p0 = smallest block, p1 = largest block (dense square blocks)
 * n = 0 means n = m.  The CSR is allocated on the device; free it with
 * pava_free_device_csr. */
typedef enum pava_gen_family {
    PAVA_GEN_STENCIL = 0,
    PAVA_GEN_BANDED = 1,
    PAVA_GEN_POWERLAW = 2,
    PAVA_GEN_BLOCKDIAG = 3
} pava_gen_family;
typedef struct pava_gen_params {
    int family;
    int m, n;
    double p0, p1, p2, p3;
} pava_gen_params;
pava_status pava_gen_device(const pava_gen_params *p, uint64_t seed, void *stream,
                            pava_csr *out);
pava_status pava_free_device_csr(pava_csr *A);

/* ---- Learned form selector ----------------------------------------------------------
 * No counterpart in the reference (which runs every format it is asked for; its only tile
 * knob is CSR5's sigma, anonymouslibHandle::setSigma, csr5/anonymouslib_avx512.h:265).
 * The selector chooses among PAVA_NVARIANTS = 32 engine forms: a kernel variant and its tile
 * parameters, the same set pava_autotune searches for one right-hand side:
 *    0 ..  3  CVR, steps 64 / 128, each with 32-bit columns and with PAVA_INDEX_AUTO
 *             (v = 2 * (steps == 128) + auto)
 *    4 .. 11  CSR5, sigma 16 / 32, default tiles per chunk or the wave-balanced count
 *             (PAVA_TILES_WAVE), 32-bit columns or PAVA_INDEX_AUTO
 *             (v = 4 + 4 * (sigma == 32) + 2 * wave + auto)
 *   12 .. 29  plain CSR row groups, lanes per row 1, 2, 4, 8, 16, 32, with 1, 4 or 16 row
 *             groups per warp tile (v = 12 + 3 * log2(lanes) + {0, 1, 2})
 *   30 .. 31  SELL, 32-bit columns or PAVA_INDEX_AUTO (v = 30 + auto); refused by matrices
 *             whose slice padding would more than double the stored elements
 * Forms fall into PAVA_NFAMILIES = 7 kernel variants (pava_variant_family): CVR 64, CVR 128,
 * CSR5 16, CSR5 32, CSR with <= 4 lanes per row, CSR with >= 8, SELL.  A matrix is described
 * by 12 structural features (pava_features); an MLP 12-64-64-32 predicts the log-time of every
 * form (so also each variant's best time, the minimum over its forms) and the smallest
 * prediction among the forms that take the matrix wins (pava_create_selected moves to the
 * next prediction when a form refuses it).  The network is trained on the GPU by the
 * library's own forward / backward / Adam kernels on timings that pava_time_variants
 * measures; exhaustive timing of all 32 forms is both the fallback and the yardstick of the
 * selector's regret. */
#define PAVA_NVARIANTS 32
#define PAVA_NFAMILIES 7
#define PAVA_TILES_WAVE (-1) /* pava_opts.tiles_per_chunk: the wave-balanced count for A */
#define PAVA_MLP_IN 12
#define PAVA_MLP_HIDDEN 64
#define PAVA_MLP_OUT 32
#define PAVA_MLP_NPARAM 7072
/* Form v's format and options (options zeroed except the form's tile parameters). */
pava_status pava_variant(int v, int *format, pava_opts *opts);
/* The kernel variant (0 .. PAVA_NFAMILIES - 1) form v belongs to, or -1 if v is out of range. */
int pava_variant_family(int v);
/* Structural features of a device CSR (sorted columns), 12 floats:
 *   0 log10 m   1 log10 nnz   2 log10 mean row length   3 row-length std / mean
 *   4 log10 max / mean row length   5 share of empty rows   6 share of nonzeros in rows
 *   longer than 64   7 share of rows with 1..4 nonzeros   8 log10(mean |col - row| / n + 1e-7)
 *   9 share of nonzeros within 64 of the diagonal   10 distinct 128-byte x lines per
 *   nonzero   11 log10(mean row span / n + 1e-7).  Integer accumulation: same bits each run. */
pava_status pava_features(const pava_csr *A, float *out12, void *stream);
/* Converts A into each of the 32 forms and times its SpMV (two warm-ups, median of `reps`
 * CUDA-event timings, x and y on the device): pava_autotune for k = 1, in form order.
 * ms[v] < 0 when form v failed; a wave-balanced CSR5 form whose tile count equals the default
 * one is the same form and gets its twin's time; *best = fastest. */
pava_status pava_time_variants(const pava_csr *A, int reps, double *ms, int *best);
typedef struct pava_mlp pava_mlp;
/* A network with He-uniform weights from `seed`, zero biases, identity normalisation. */
pava_status pava_mlp_create(uint64_t seed, pava_mlp **out);
/* Parameters (PAVA_MLP_NPARAM floats: W1[64][12] b1 W2[64][64] b2 W3[32][64] b3) and the
 * feature normalisation (x - mean) / std applied to every batch; any pointer may be NULL.
 * Setting parameters resets the Adam state. */
pava_status pava_mlp_get_params(const pava_mlp *m, float *params, float *mean12, float *std12);
pava_status pava_mlp_set_params(pava_mlp *m, const float *params, const float *mean12,
                                const float *std12);
/* Uploads a batch: B x 12 raw features, optional B x 32 targets and 0/1 mask (NULL mask = all
 * ones).  The loss is the masked mean squared error. */
pava_status pava_mlp_set_batch(pava_mlp *m, int B, const float *X, const float *T,
                               const float *mask);
/* Outputs for the current batch (B x 32, host). */
pava_status pava_mlp_forward(pava_mlp *m, float *Y);
/* Gradient of the loss w.r.t. the parameters (PAVA_MLP_NPARAM floats, host) and the loss. */
pava_status pava_mlp_gradient(pava_mlp *m, float *grad, float *loss);
/* `epochs` full-batch Adam steps (beta 0.9 / 0.999, eps 1e-8) on the current batch;
 * loss_hist (may be NULL) receives the loss before each step. */
pava_status pava_mlp_train(pava_mlp *m, int epochs, float lr, float *loss_hist);
pava_status pava_mlp_destroy(pava_mlp *m);
/* The form the network predicts fastest for a device CSR (and the 32 predictions), whether
 * or not that form takes the matrix.  Uses the network's batch slot (a 1-sample batch
 * replaces the current one). */
pava_status pava_select(pava_mlp *m, const pava_csr *A, int *variant, float *pred32);
/* pava_create with the selected form: by the network when m != NULL and A is on the
 * device (the predictions in order, past any form that refuses the matrix), otherwise by
 * timing all 32 (the exhaustive fallback). */
pava_status pava_create_selected(const pava_csr *A, pava_mlp *m, void *stream,
                                 pava_handle **out, int *variant);

/* COO -> CSR on the device: the loader's conversion (readCOOMatrix's symmetric expansion and
 * 1-based shift, utils/basicMatrix.cpp:63-253; convertCOO2CSR via mkl_dcsrcoo, :350-415).
 * rows / cols / vals are device arrays of nnz entries with index base 0 or 1; symmetric = 1
 * adds (c, r) for every off-diagonal (r, c).  The result has ascending rows and ascending
 * columns inside each row, duplicates kept as separate entries in input order (the same as
 * pava_coo_to_csr of pava_host.h); it is allocated on the device -- free it with
 * pava_free_device_csr.  Indices outside the matrix give PAVA_E_INVALID_CSR. */
pava_status pava_coo_to_csr_device(int m, int n, long long nnz, const int *rows,
                                   const int *cols, const double *vals, int index_base,
                                   int symmetric, void *stream, pava_csr *out);

/* Drop-ins for the reference's engine entry points, same signatures and meaning:
 * conduct_cvr (cvr/cvr.h:1953) and conduct_csr5 (csr5/csr5.h:72-74).  Each copies the CSR to
 * the device, converts (timed as the convert column), runs one SpMV into refOut / y (the
 * checked result), times numIterations more, and prints the reference's line
 * " Performance <name> CVR|CSR5 <SMs> <convert s> <exec s>" (utils/basicMatrix.cpp:491-495).
 * Returns 0 on success or a pava_status.  alpha is accepted and, as in the reference, not
 * applied (cvr/cvr.h never reads it; csr5_spmv_avx512.h comments out its multiply). */
/* What one benchmark section measured (pava_conduct): the reference prints it as
 * " Performance ..." and keeps nothing (utils/basicMatrix.cpp:491-495). */
typedef struct pava_run_record {
    int status;              /* pava_status of the section */
    int format, precision, index_mode;
    int steps, sigma, tiles_per_chunk, lanes_per_row;  /* the form's tile parameters */
    int sm_count, iterations;
    long long chunks;
    double convert_s;        /* device time of the conversion */
    double exec_s;           /* seconds per timed SpMV (-1 if none ran) */
    double alg_bytes;        /* compulsory bytes of one SpMV */
    double format_bytes;     /* bytes one SpMV streams from the format plus x and y */
} pava_run_record;

/* One benchmark section on a host CSR (the body of conduct_cvr_gpu / conduct_csr5_gpu, for any
 * format and options): convert, the checked first SpMV into y, `iterations` timed SpMVs, the
 * Performance line; `rec` (may be NULL) receives the measurements.  opts NULL = the drop-ins'
 * defaults (16-bit column offsets where they fit). */
int pava_conduct(int format, const pava_csr *A, const double *x, double *y, const char *name,
                 int iterations, const pava_opts *opts, pava_run_record *rec);

int conduct_cvr_gpu(int numRows, int numCols, int nItems_raw, int *h_rowDelimiters,
                    int *h_cols, double *h_val, double *h_vec, double *refOut, int alpha,
                    char *matrixName, int numIterations);
int conduct_csr5_gpu(int m, int n, int nnzA, int *csrRowPtrA, int *csrColIdxA,
                     double *csrValA, double *x, double *y, double alpha, char *matrixName,
                     int numIterations);

#ifdef __cplusplus
}
#endif
#endif /* PAVA_GPU_H */
