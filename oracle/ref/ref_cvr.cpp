/*
 * Test infrastructure (oracle only).  Compiles the reference's CVR engine (cvr/cvr.h) from the
 * reference tree and exposes it as plain C functions for the parity tests and the timed CPU
 * baseline.  Nothing in the product links this file.
 *
 * It calls pre_processing (cvr/cvr.h:583) and spmv_compute_kernel (cvr/cvr.h:1062) directly,
 * with the buffers conduct_cvr (cvr/cvr.h:1953-2030) allocates, because conduct_cvr has no
 * return statement (undefined behaviour under optimisation).  Differences from conduct_cvr,
 * all needed to run the reference safely and to use it as an oracle:
 *   - nnz is padded to a multiple of 16 (cvr/cvr.h:1958); the padding elements are value 0,
 *     column 0, and belong to the last row (as utils/basicMatrix.cpp:150,211-216 pads the COO
 *     input of the reference benchmark), so row_ptr[m] is the padded count;
 *   - every array gets zeroed slack, because the engine prefetches past its chunk
 *     (cvr/cvr.h:1306) and gathers up to the padded count (cvr/cvr.h:1009);
 *   - y is zeroed before the first call, and only the first call is returned: later calls add
 *     into rows shared between threads without clearing them (cvr/cvr.h:1415,1717,1855).
 */
#include <omp.h>
#include <string.h>
#include <stdlib.h>
#include "cvr/cvr.h"

/* utils/basicMatrix.cpp:491 needs MKL; conduct_cvr references it, this file never calls it. */
int printPerformance(char *, char *, int, double, double) { return 0; }

static double wall_s() { return microtime(); }

template <class T> static T *zalloc(size_t n) {
    T *p = (T *)_mm_malloc(sizeof(T) * (n ? n : 1), 64);
    if (p) memset(p, 0, sizeof(T) * (n ? n : 1));
    return p;
}

struct CvrRefState {
    int nthreads, m, n, nitems;
    int *rp, *ci;
    double *v;
    double *vals, *x;
    int *cols, *fin, *fin2, *rec, *split, *nblock, *nnz_rows;
    size_t rec_len;
};

static void cvr_free(CvrRefState *s) {
    _mm_free(s->rp); _mm_free(s->ci); _mm_free(s->v); _mm_free(s->vals); _mm_free(s->cols);
    _mm_free(s->fin); _mm_free(s->fin2); _mm_free(s->rec); _mm_free(s->x);
    free(s->split); free(s->nblock); _mm_free(s->nnz_rows);
}

static int cvr_setup(CvrRefState *s, int nthreads, int m, int n, int nnz, const int *rp,
                     const int *ci, const double *v, const double *x) {
    memset(s, 0, sizeof(*s));
    s->nthreads = nthreads; s->m = m; s->n = n;
    const int nitems = (nnz % 16 == 0) ? nnz : (nnz + 16) / 16 * 16; /* cvr/cvr.h:1958 */
    s->nitems = nitems;
    const size_t slack = 256;
    s->rp = zalloc<int>((size_t)m + 1 + slack);
    s->ci = zalloc<int>((size_t)nitems + slack);
    s->v = zalloc<double>((size_t)nitems + slack);
    s->x = zalloc<double>((size_t)n + slack);
    if (!s->rp || !s->ci || !s->v || !s->x) return -1;
    memcpy(s->rp, rp, sizeof(int) * (size_t)m);
    for (size_t i = (size_t)m; i < (size_t)m + 1 + slack; i++) s->rp[i] = nitems;
    memcpy(s->ci, ci, sizeof(int) * (size_t)nnz);
    memcpy(s->v, v, sizeof(double) * (size_t)nnz);
    memcpy(s->x, x, sizeof(double) * (size_t)n);
    const int omega = 1; /* cvr/cvr.h:1974 */
    s->vals = zalloc<double>((size_t)nitems + slack);
    s->cols = zalloc<int>((size_t)nitems + slack);
    s->fin = zalloc<int>((size_t)16 * nthreads + slack);
    s->fin2 = zalloc<int>((size_t)16 * omega * nthreads + slack);
    s->rec_len = (size_t)2 * ((size_t)m + 240 + (size_t)nthreads * 32) + slack;
    s->rec = zalloc<int>(s->rec_len);
    s->split = (int *)calloc((size_t)nthreads * 2 + 16, sizeof(int));
    s->nblock = (int *)calloc((size_t)nthreads + 16, sizeof(int));
    s->nnz_rows = zalloc<int>((size_t)4 * nthreads + slack);
    if (!s->vals || !s->cols || !s->fin || !s->fin2 || !s->rec || !s->split || !s->nblock ||
        !s->nnz_rows)
        return -1;
    for (int i = 0; i < nthreads; i++) s->nblock[i] = 1;
    return 0;
}

extern "C" {

/* Runs the reference CVR conversion once and the CVR SpMV once into zeroed y (the oracle
 * output, y has m entries), then `iters` more timed SpMV calls into a scratch vector.
 * convert_s / exec_s receive wall seconds for the conversion and per timed call (as
 * cvr/cvr.h:2076-2112 measure them).  Optional outputs (NULL to skip) expose the CVR
 * arrays: vals/cols (padded count), records (rec_len ints), split (2*T), nnz_rows (4*T),
 * final_2 (16*T).  Returns 0, or -1 on allocation failure. */
int pava_ref_cvr(int nthreads, int m, int n, int nnz, const int *rp, const int *ci,
                 const double *v, const double *x, double *y, int iters, double *convert_s,
                 double *exec_s, double *out_vals, int *out_cols, int *out_rec,
                 long long out_rec_len, int *out_split, int *out_nnz_rows, int *out_final2) {
    CvrRefState s;
    if (cvr_setup(&s, nthreads, m, n, nnz, rp, ci, v, x) != 0) { cvr_free(&s); return -1; }
    /* front slack: records written at step 0 of a stealing lane carry row -1
     * (cvr/cvr.h:933-937) and the first SpMV stores to y[-1] (cvr/cvr.h:1447-1452). */
    double *ybase = zalloc<double>((size_t)m + 512);
    double *ybase2 = zalloc<double>((size_t)m + 512);
    double *yout = ybase + 256;
    double *yit = ybase2 + 256;
    char name[8] = "oracle";
    const int omega = 1;
    double t1 = wall_s();
    pre_processing(nthreads, 0, nthreads, s.nblock, s.rec, s.nnz_rows, s.vals, s.cols, s.v, s.ci,
                   s.fin, s.fin2, s.split, yout, s.nitems, m, omega, s.rp, name);
    double t2 = wall_s();
    spmv_compute_kernel(nthreads, 0, nthreads, s.nblock, s.rec, s.nnz_rows, s.vals, s.cols, s.v,
                        s.ci, s.fin, s.fin2, s.split, yout, s.nitems, m, omega, s.rp, name, s.x, 1);
    memcpy(y, yout, sizeof(double) * (size_t)m);
    double t3 = wall_s(), t4 = t3;
    if (iters > 0) {
        spmv_compute_kernel(nthreads, 0, nthreads, s.nblock, s.rec, s.nnz_rows, s.vals, s.cols,
                            s.v, s.ci, s.fin, s.fin2, s.split, yit, s.nitems, m, omega, s.rp, name,
                            s.x, iters);
        t4 = wall_s();
    }
    if (convert_s) *convert_s = t2 - t1;
    if (exec_s) *exec_s = iters > 0 ? (t4 - t3) / iters : 0.0;
    if (out_vals) memcpy(out_vals, s.vals, sizeof(double) * (size_t)s.nitems);
    if (out_cols) memcpy(out_cols, s.cols, sizeof(int) * (size_t)s.nitems);
    if (out_rec) {
        size_t nrec = (size_t)out_rec_len < s.rec_len ? (size_t)out_rec_len : s.rec_len;
        memcpy(out_rec, s.rec, sizeof(int) * nrec);
    }
    if (out_split) memcpy(out_split, s.split, sizeof(int) * 2 * (size_t)nthreads);
    if (out_nnz_rows) memcpy(out_nnz_rows, s.nnz_rows, sizeof(int) * 4 * (size_t)nthreads);
    if (out_final2) memcpy(out_final2, s.fin2, sizeof(int) * 16 * (size_t)nthreads);
    _mm_free(ybase); _mm_free(ybase2);
    cvr_free(&s);
    return 0;
}

/* Length of the record array the reference allocates (cvr/cvr.h:2024), for sizing out_rec. */
long long pava_ref_cvr_record_len(int nthreads, int m) {
    return (long long)2 * ((long long)m + 240 + (long long)nthreads * 32) + 256;
}

} /* extern "C" */
