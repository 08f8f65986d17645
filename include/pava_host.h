/*
 * pava_host.h -- host-side C ABI of the pava benchmark surface: seeded synthetic matrix
 * generators (the inputs of the benchmark configurations), Matrix Market I/O and COO -> CSR.
 *
 * These replace the reference's loader and conversion (readCOOMatrix,
 * utils/basicMatrix.cpp:63-253; convertCOO2CSR via mkl_dcsrcoo, utils/basicMatrix.cpp:350-415;
 * initVectors, utils/basicMatrix.cpp:499-520).  All generators are deterministic functions of
 * (seed, row, element): counter-based random numbers, so any thread count gives the same
 * matrix.  Every function returns 0 on success and a negative pava_status on failure.
 */
#ifndef PAVA_HOST_H
#define PAVA_HOST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- generators: two calls, row lengths first (fill rp[0..m], return nnz via rp[m]), then
 *      the columns and values into caller-allocated arrays of rp[m] entries ---------------- */

/* 2-D 5-point Laplacian on a grid x grid mesh, rows in natural order, sorted columns,
 * diagonal 4, off-diagonals -1. */
int pava_gen_laplace2d_rowptr(int grid, int *rp);
int pava_gen_laplace2d_fill(int grid, const int *rp, int *ci, double *v);

/* Power-law rows: a row is empty with probability p_empty, else its length is
 * clamp(round(exp(N(mu, sigma))), 1, cap) with mu = ln(mean) - sigma^2/2; columns uniform in
 * [0, n) without duplicates, sorted; values N(0, 1). */
int pava_gen_powerlaw_rowptr(int m, int n, double mean, double sigma, int cap, double p_empty,
                             uint64_t seed, int *rp);
int pava_gen_powerlaw_fill(int m, int n, uint64_t seed, const int *rp, int *ci, double *v);

/* 3-D 27-point stencil on a grid^3 mesh: off-diagonals U[-1, 0), diagonal 1.01 x the row's
 * absolute off-diagonal sum; every value is exactly representable in FP32. */
int pava_gen_stencil27_rowptr(int grid, int *rp);
int pava_gen_stencil27_fill(int grid, uint64_t seed, const int *rp, int *ci, double *v);

/* Banded: per_row distinct columns uniform in [r - halfbw, r + halfbw] clipped to [0, m),
 * sorted; values N(0, 1). */
int pava_gen_banded_rowptr(int m, int halfbw, int per_row, int *rp);
int pava_gen_banded_fill(int m, int halfbw, uint64_t seed, const int *rp, int *ci, double *v);

/* Random: row lengths Poisson(mean) clipped to [0, n), columns uniform without duplicates,
 * sorted; values N(0, 1). */
int pava_gen_random_rowptr(int m, int n, double mean, uint64_t seed, int *rp);
int pava_gen_random_fill(int m, int n, uint64_t seed, const int *rp, int *ci, double *v);

/* Block diagonal: dense square blocks of sizes uniform in [bmin, bmax] down the diagonal;
 * values N(0, 1). */
int pava_gen_blockdiag_rowptr(int m, int bmin, int bmax, uint64_t seed, int *rp);
int pava_gen_blockdiag_fill(int m, uint64_t seed, const int *rp, int *ci, double *v);

/* x[i] = lo + (hi - lo) * U(seed, i); with fp32 != 0 every entry is rounded to FP32 first
 * (so that an FP32 copy is exact). */
int pava_gen_uniform(int n, double lo, double hi, uint64_t seed, int fp32, double *x);

/* initVectors (utils/basicMatrix.cpp:499-520): y = 0, y_ref = 0, x[i] = i % 3 (NULL skips). */
void pava_init_vectors(int m, int n, double *x, double *y, double *y_ref);

/* ---- Matrix Market --------------------------------------------------------------------- */

/* Reads the banner and size line.  nnz_alloc is the number of COO entries the reader will
 * produce (twice the stored count for symmetric / skew / hermitian files, which are
 * expanded).  kind: 0 real, 1 integer, 2 pattern, 3 complex (real part kept). */
int pava_mtx_info(const char *path, int *m, int *n, long long *nnz_alloc, int *kind,
                  int *symmetric);

/* Reads the entries as 0-based COO (the file is 1-based; the reference's loader passes the
 * 1-based indices to a 0-based conversion, utils/basicMatrix.cpp:361,384, which shifts every
 * row and column by one -- this reader converts explicitly).  *nnz receives the count. */
int pava_mtx_read(const char *path, int *rows, int *cols, double *vals, long long *nnz);

/* Writes a CSR matrix as "matrix coordinate real general", 1-based, %.17g values. */
int pava_mtx_write(const char *path, int m, int n, const int *rp, const int *ci,
                   const double *v);

/* COO -> CSR, rows and columns sorted; duplicates are kept as separate entries. */
int pava_coo_to_csr(int m, int n, long long nnz, const int *rows, const int *cols,
                    const double *vals, int *rp, int *ci, double *v);

#ifdef __cplusplus
}
#endif
#endif /* PAVA_HOST_H */
