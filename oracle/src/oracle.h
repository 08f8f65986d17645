/*
 * ORACLE -- test infrastructure only.  A plain-C restatement of the reference's CVR and CSR5
 * engines (cvr/cvr.h, csr5/) plus a long-double CSR reference and error metrics.  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark use it, as the oracle the
 * GPU results are compared with or as the reported CPU number; the product never links or calls it.
 *
 * Parity pin: every function here is checked in the CPU test suite against the reference
 * itself, compiled from the reference tree into oracle/_ref (see oracle/Makefile), and against
 * the committed golden fixtures under tests/golden/ that were generated from it.
 */
#ifndef PAVA_ORACLE_H
#define PAVA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- CSR reference and error metric ------------------------------------------------------ */

/* y_ref[i] = sum_j a_ij x_j accumulated in long double, rounded to double once; absum[i] =
 * sum_j |a_ij x_j| (may be NULL).  Follows referenceSpMV (utils/basicMatrix.cpp:538-556)
 * with a wider accumulator. */
void oracle_csr_ref(int m, const int *rp, const int *ci, const double *v, const double *x,
                    double *y_ref, double *absum);

/* Per-row relative error rel_i = |y_i - yref_i| / max(|yref_i|, absum_i) (absolute when both
 * are 0).  Writes max and mean over rows; returns the number of rows with rel_i > tol. */
long long oracle_rel_error(int m, const double *y, const double *y_ref, const double *absum,
                           double tol, double *max_rel, double *mean_rel);

/* checkResults (utils/basicMatrix.cpp:559-587): rows with |y_ref - y| > 0.01 |y_ref|. */
long long oracle_check_results(int m, const double *y, const double *y_ref);

/* ---- CVR restatement (cvr/cvr.h, 8 SIMD lanes, omega = 1) -------------------------------- */

/* Sizes a CVR layout for T threads: padded element count and record-array length, as
 * conduct_cvr allocates them (cvr/cvr.h:1958, 2024). */
int oracle_cvr_padded(int nnz);
long long oracle_cvr_record_len(int nthreads, int m);

/* CSR -> CVR (pre_processing, cvr/cvr.h:583-1060) on a CSR whose nnz is already padded to a
 * multiple of 16 with the padding in the last row (rp[m] == nitems).  rp must have 2 slack
 * entries past m equal to rp[m]; vals/cols/h_val/h_cols need 64 zeroed slack entries.  Outputs
 * vals/cols (nitems), rec (record_len, zero-initialised by the caller), split (2T, zeroed),
 * nnz_rows (4T), final2 (16T). */
void oracle_cvr_convert(int nthreads, int m, int nitems, const int *rp, const int *h_cols,
                        const double *h_val, double *vals, int *cols, int *rec, int *split,
                        int *nnz_rows, int *final2);

/* CVR SpMV (spmv_compute_kernel, cvr/cvr.h:1062-1884), first call into y (m + 2 entries,
 * zeroed by the caller: the engine never writes empty rows). */
void oracle_cvr_spmv(int nthreads, int m, int nitems, const double *vals, const int *cols,
                     const int *rec, const int *split, const int *nnz_rows, const int *final2,
                     const double *x, double *y);

/* ---- CSR5 restatement (csr5/, omega = 8) ------------------------------------------------- */

typedef struct {
    int sigma, omega, p, bit_y_offset, bit_scansum_offset, num_packet, num_offsets;
    int tail_partition_start;
} oracle_csr5_info;

/* Fills the tile parameters asCSR5 derives (csr5/anonymouslib_avx512.h:118-139). */
void oracle_csr5_params(int nnz, int sigma, oracle_csr5_info *info);

/* CSR -> CSR5 (generate_partition_pointer, generate_partition_descriptor,
 * generate_partition_descriptor_offset, aosoa_transpose; csr5/detail/avx512/format_avx512.h).
 * tile_ptr (p+1), tile_desc (p*8*num_packet, zeroed by caller), desc_off_ptr (p+1, zeroed);
 * returns num_offsets.  Call oracle_csr5_offsets afterwards when num_offsets > 0.  cols/vals
 * (nnz) are transposed out of place into tcols/tvals. */
int oracle_csr5_convert(int m, int nnz, const int *rp, const int *cols, const double *vals,
                        const oracle_csr5_info *info, unsigned *tile_ptr, unsigned *tile_desc,
                        int *desc_off_ptr, int *tcols, double *tvals);
void oracle_csr5_offsets(const int *rp, const oracle_csr5_info *info, const unsigned *tile_ptr,
                         const unsigned *tile_desc, const int *desc_off_ptr, int *desc_off);

/* CSR5 SpMV (csr5_spmv, csr5/detail/avx512/csr5_spmv_avx512.h:346-382), first call into y
 * (zeroed by caller), with `nthreads` static chunks of tiles as the reference's OpenMP loop
 * schedules them (csr5_spmv_avx512.h:70,102). */
void oracle_csr5_spmv(int nthreads, int m, const int *rp, const int *ocols, const double *ovals,
                      const int *tcols, const double *tvals, const oracle_csr5_info *info,
                      const unsigned *tile_ptr, const unsigned *tile_desc,
                      const int *desc_off_ptr, const int *desc_off, const double *x, double *y);

/* One-call conveniences: convert + first SpMV; they allocate internally.  The CVR one pads nnz
 * to a multiple of 16 into the last row first.  Return 0 or -1 on allocation failure. */
int oracle_cvr_run(int nthreads, int m, int n, int nnz, const int *rp, const int *ci,
                   const double *v, const double *x, double *y, double *convert_s,
                   double *exec_s, int iters);
int oracle_csr5_run(int nthreads, int sigma, int m, int n, int nnz, const int *rp,
                    const int *ci, const double *v, const double *x, double *y,
                    double *convert_s, double *exec_s, int iters);

#ifdef __cplusplus
}
#endif
#endif
