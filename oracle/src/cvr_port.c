/*
 * ORACLE -- test infrastructure only (never linked by the product).
 *
 * Scalar restatement of the reference CVR engine, cvr/cvr.h: the CSR->CVR conversion
 * pre_processing (cvr/cvr.h:583-1060) and the CVR SpMV spmv_compute_kernel
 * (cvr/cvr.h:1062-1884), for T threads of 8 SIMD lanes, omega = 1, one row block per thread
 * (conduct_cvr, cvr/cvr.h:1974-2004).  The 16-lane AVX-512 registers are modelled as arrays of
 * 16 ints / 8 doubles with the same masking, so the layout (values, columns, records, split,
 * final_2) is reproduced bit for bit.  Threads run one after another, so rows shared by two
 * threads see their writes in thread order (the reference races on them and relies on y
 * being zero before the first call, cvr/cvr.h:1413-1421).
 *
 * Quirks kept as the reference has them:
 *   - a record written at step 0 in the stealing branch carries the lane's flag value, which
 *     is -1 before any steal (cvr/cvr.h:933-937); the first SpMV then writes y[-1]
 *     (cvr/cvr.h:1447-1452), so callers give y one slot of front slack;
 *   - final_2 snapshots lane row ids, including 0 for lanes that never held a row, and the
 *     final write-out stores into y[final_2[k]] (cvr/cvr.h:1840-1868): a thread whose chunk
 *     spans eight rows or fewer writes 0 into y[0].  Tests use matrices where every thread
 *     spans more than eight rows.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include "oracle.h"

int oracle_cvr_padded(int nnz) { return (nnz % 16 == 0) ? nnz : (nnz + 16) / 16 * 16; }

long long oracle_cvr_record_len(int nthreads, int m) {
    return (long long)2 * ((long long)m + 240 + (long long)nthreads * 32) + 256;
}

/* Thread chunk [s, e) of the padded element range (cvr/cvr.h:602-645). */
static void cvr_chunk(int T, int nitems, int t, int *s, int *e) {
    int thread_nnz = (nitems / T / 16) * 16;
    int thread_break = (nitems - thread_nnz * T) / 16;
    if (t < thread_break) {
        *s = t * (thread_nnz + 16);
        *e = (t + 1) * (thread_nnz + 16);
    } else {
        *s = t * thread_nnz + thread_break * 16;
        *e = (t + 1) * thread_nnz + thread_break * 16;
    }
    if (t == T - 1) *e = nitems;
}

/* Row range of a chunk by the two binary searches of cvr/cvr.h:666-717. */
static void cvr_rows(const int *rp, int m, int s, int e, int *rs, int *re) {
    int start = 0, stop = m, med;
    while (stop >= start) {
        med = (stop + start) / 2;
        if (s >= rp[med]) start = med + 1; else stop = med - 1;
    }
    *rs = start - 1;
    start = *rs;
    stop = m;
    while (stop >= start) {
        med = (stop + start) / 2;
        if ((e - 1) >= rp[med]) start = med + 1; else stop = med - 1;
    }
    int r = start - 1;
    while ((rp[r + 1] - rp[r] == 0) && (r <= m)) r++;
    *re = r;
}

void oracle_cvr_convert(int T, int m, int nitems, const int *rp, const int *h_cols,
                        const double *h_val, double *vals_all, int *cols_all, int *rec_all,
                        int *split, int *nnz_rows, int *final2_all) {
    for (int t = 0; t < T; t++) {
        int s, e, rs, re;
        cvr_chunk(T, nitems, t, &s, &e);
        cvr_rows(rp, m, s, e, &rs, &re);
        nnz_rows[t * 4 + 0] = s;
        nnz_rows[t * 4 + 1] = e;
        nnz_rows[t * 4 + 2] = rs;
        nnz_rows[t * 4 + 3] = re;
        const int span = re - rs + 1;
        double *vals = vals_all + s;
        int *cols = cols_all + s;
        const double *ov = h_val + s;
        const int *oc = h_cols + s;
        int *final2 = final2_all + t * 16;
        int *rec = rec_all + 2 * (t * 32 + rs) / 16 * 16;
        int seg = 0;

        int valID[16], rowID[16], count[16], flag[16], first_flag[16];
        for (int k = 0; k < 16; k++) {
            valID[k] = 0; rowID[k] = 0; count[k] = 1; flag[k] = -1; first_flag[k] = 0;
        }
        const int rs_init = rs;
        for (int i = 0; i < 8; i++) { /* cvr/cvr.h:756-788 */
            if (rs < re) {
                valID[i] = rp[rs] - s; rowID[i] = rs; count[i] = rp[rs + 1] - rp[rs];
            } else if (rs == re) {
                valID[i] = rp[rs] - s; rowID[i] = rs; count[i] = e - rp[rs];
            } else {
                valID[i] = 0; rowID[i] = 0; count[i] = 0;
            }
            if (i == 0) {
                valID[i] = 0;
                count[i] = rp[rs + 1] - s;
                if (rs == re) count[i] = e - s;
            }
            rs++;
        }
        int first_in = 0;
        const int nsteps = (e - s) / 8;
        for (int i = 0; i < nsteps; i++) {
            int xx = count[0];
            for (int k = 1; k < 8; k++) xx = count[k] < xx ? count[k] : xx;
            if (xx == 0) {
                for (int kk = 0; kk < 8; kk++) {
                    if (count[kk] != 0) continue;
                    if (rs <= re) { /* rows branch, cvr/cvr.h:857-905 */
                        if (rowID[kk] == rs_init) {
                            split[t * 2] = i * 8 + kk;
                        } else {
                            rec[seg] = i * 8 + kk;
                            rec[seg + 1] = rowID[kk];
                            seg += 2;
                        }
                        while (rp[rs + 1] - rp[rs] == 0) rs++;
                        valID[kk] = rp[rs] - s;
                        rowID[kk] = rs;
                        count[kk] = rp[rs + 1] - rp[rs];
                        if (rs == re) {
                            if (split[t * 2 + 1] == 0) split[t * 2 + 1] = i * 8 + kk;
                            count[kk] = e - rp[rs];
                            for (int k = 0; k < 8; k++) final2[k] = rowID[k];
                            for (int k = 0; k < 16; k++)
                                if (count[k] == 0) flag[k] = 0;
                        }
                        rs++;
                    } else { /* stealing branch, cvr/cvr.h:906-989 */
                        int tot = 0;
                        for (int k = 0; k < 8; k++) tot += count[k];
                        int ave = tot / 8;
                        int cali = 0;
                        for (cali = 0; cali < 8; cali++)
                            if (count[cali] > ave) break;
                        if (first_flag[kk] == 0) {
                            if (first_in == 0) {
                                if (split[t * 2 + 1] == 0)
                                    split[t * 2 + 1] = (span <= 8) ? -1 : i * 8 + kk;
                                for (int k = 0; k < 8; k++) final2[k] = rowID[k];
                                first_in = 1;
                            }
                            if (i != 0) {
                                rec[seg] = i * 8 + kk;
                                rec[seg + 1] = kk;
                                flag[kk] = cali;
                                first_flag[kk] = 1;
                            } else {
                                rec[seg] = i * 8 + kk;
                                rec[seg + 1] = flag[kk];
                                flag[kk] = cali;
                            }
                        } else {
                            rec[seg] = i * 8 + kk;
                            rec[seg + 1] = flag[kk];
                            flag[kk] = cali;
                        }
                        valID[kk] = valID[cali];
                        rowID[kk] = cali;
                        count[kk] = ave;
                        count[cali] = count[cali] - ave;
                        valID[cali] = valID[cali] + ave;
                        seg += 2;
                    }
                }
            }
            /* gather into lane-interleaved order, cvr/cvr.h:1009-1023 */
            for (int k = 0; k < 8; k++) {
                vals[i * 8 + k] = ov[valID[k]];
                cols[i * 8 + k] = oc[valID[k]];
            }
            for (int k = 0; k < 8; k++) { valID[k] += 1; count[k] -= 1; }
            for (int k = 8; k < 16; k++) { valID[k] = 0; count[k] = 0; }
            if (i == nsteps - 1) { /* terminal records, cvr/cvr.h:1028-1045 */
                for (int kk = 0; kk < 8; kk++) {
                    rec[seg] = -1;
                    rec[seg + 1] = (flag[kk] == -1) ? kk : flag[kk];
                    seg += 2;
                }
            }
        }
    }
}

/* One 8-lane step: z[k] = fma(v, x[c], z[k]) (cvr/cvr.h:1341-1345). */
static inline void cvr_fma_step(const double *v, const int *c, const double *x, double *z) {
    for (int k = 0; k < 8; k++) z[k] = fma(v[k], x[c[k]], z[k]);
}

void oracle_cvr_spmv(int T, int m, int nitems, const double *vals_all, const int *cols_all,
                     const int *rec_all, const int *split, const int *nnz_rows,
                     const int *final2_all, const double *x, double *y) {
    (void)m; (void)nitems;
    for (int t = 0; t < T; t++) {
        const int s = nnz_rows[t * 4], e = nnz_rows[t * 4 + 1];
        const int rs = nnz_rows[t * 4 + 2], re = nnz_rows[t * 4 + 3];
        int cut_last = 0, cut_next = 0;
        if (t == 0) {
            cut_next = (nnz_rows[(t + 1) * 4 + 2] == re);
        } else if (t == T - 1) {
            cut_last = (nnz_rows[(t - 1) * 4 + 3] == rs);
        } else {
            cut_next = (nnz_rows[(t + 1) * 4 + 2] == re);
            cut_last = (nnz_rows[(t - 1) * 4 + 3] == rs);
        }
        const double *v = vals_all + s;
        const int *c = cols_all + s;
        const int *final2 = final2_all + t * 16;
        const int *rec = rec_all + 2 * (t * 32 + rs) / 16 * 16;
        double z[8] = {0}, tr[16] = {0};
        int seg = 0, t_index = 0, i;
        const int ncsr_start = split[t * 2], ncsr = split[t * 2 + 1];
        const int len = e - s;

        /* steps before the thread's first row ends (cvr/cvr.h:1264-1351) */
        for (i = 0; i < ncsr_start / 8 * 8; i += 8) {
            while ((rec[seg] & (int)0xfffffff8) == (i & (int)0xfffffff8)) {
                int lane = rec[seg] & 7;
                y[rec[seg + 1]] = z[lane] + 0.0;
                z[lane] = 0.0;
                seg += 2;
            }
            cvr_fma_step(v + i, c + i, x, z);
        }
        /* the step of the first row's end (cvr/cvr.h:1357-1505) */
        for (i = ncsr_start / 8 * 8; i < ncsr_start / 8 * 8 + 8; i += 8) {
            int lane0 = ncsr_start % 8;
            if (cut_last) y[rs] += z[lane0] + 0.0;
            else y[rs] = z[lane0] + 0.0;
            z[lane0] = 0.0;
            if (ncsr_start == ncsr)
                for (int k = 0; k < 16; k++) tr[k] = 0.0;
            while ((rec[seg] & (int)0xfffffff8) == (i & (int)0xfffffff8)) {
                int lane = rec[seg] & 7;
                if (ncsr_start != ncsr) y[rec[seg + 1]] = z[lane] + 0.0;
                else tr[rec[seg + 1]] = z[lane] + 0.0;
                z[lane] = 0.0;
                seg += 2;
            }
            cvr_fma_step(v + i, c + i, x, z);
        }
        /* steady state (cvr/cvr.h:1512-1598) */
        for (i = ncsr_start / 8 * 8 + 8; i < ncsr / 8 * 8; i += 8) {
            while ((rec[seg] & (int)0xfffffff8) == (i & (int)0xfffffff8)) {
                int lane = rec[seg] & 7;
                y[rec[seg + 1]] = z[lane];
                z[lane] = 0.0;
                seg += 2;
            }
            cvr_fma_step(v + i, c + i, x, z);
        }
        /* the step where the last row was taken or stealing began (cvr/cvr.h:1605-1757) */
        if (ncsr >= 0 && (ncsr / 8 != ncsr_start / 8)) {
            for (i = ncsr / 8 * 8; i < ncsr / 8 * 8 + 8; i += 8) {
                while ((rec[seg] & (int)0xfffffff8) == (i & (int)0xfffffff8)) {
                    int lane = rec[seg] & 7;
                    if (rec[seg] <= ncsr) {
                        y[rec[seg + 1]] = z[lane];
                        z[lane] = 0.0;
                        seg += 2;
                    } else if (t_index != -1) {
                        t_index = -1;
                        tr[lane] += z[lane];
                        z[lane] = 0.0;
                    } else {
                        tr[rec[seg + 1]] += z[lane];
                        z[lane] = 0.0;
                        seg += 2;
                    }
                }
                cvr_fma_step(v + i, c + i, x, z);
            }
        }
        /* tail: partial sums go to the temporary slots (cvr/cvr.h:1767-1821) */
        for (i = ncsr / 8 * 8 + 8; i < len; i += 8) {
            while ((rec[seg] & (int)0xfffffff8) == (i & (int)0xfffffff8)) {
                int lane = rec[seg] & 7;
                tr[rec[seg + 1]] += z[lane];
                z[lane] = 0.0;
                seg += 2;
            }
            cvr_fma_step(v + i, c + i, x, z);
        }
        if (i == len) { /* terminal records and final write-out (cvr/cvr.h:1823-1868) */
            for (int k = 0; k < 8; k++) {
                tr[rec[seg + 1]] += z[k];
                seg += 2;
            }
            for (int k = 0; k < 8; k++) {
                int w = final2[k];
                if ((w == re && cut_next) || (w == rs && cut_last)) y[w] += tr[k];
                else y[w] = tr[k];
            }
        }
    }
}

static double now_s(void) {
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + tv.tv_usec / 1e6;
}

int oracle_cvr_run(int T, int m, int n, int nnz, const int *rp, const int *ci, const double *v,
                   const double *x, double *y, double *convert_s, double *exec_s, int iters) {
    const int nitems = oracle_cvr_padded(nnz);
    const size_t slack = 256;
    int *rp2 = (int *)calloc((size_t)m + 1 + slack, sizeof(int));
    int *ci2 = (int *)calloc((size_t)nitems + slack, sizeof(int));
    double *v2 = (double *)calloc((size_t)nitems + slack, sizeof(double));
    double *vals = (double *)calloc((size_t)nitems + slack, sizeof(double));
    int *cols = (int *)calloc((size_t)nitems + slack, sizeof(int));
    long long rl = oracle_cvr_record_len(T, m);
    int *rec = (int *)calloc((size_t)rl, sizeof(int));
    int *split = (int *)calloc((size_t)T * 2 + 16, sizeof(int));
    int *nnz_rows = (int *)calloc((size_t)T * 4 + 16, sizeof(int));
    int *final2 = (int *)calloc((size_t)T * 16 + 16, sizeof(int));
    double *ybuf = (double *)calloc((size_t)m + 2 * slack, sizeof(double));
    int rc = -1;
    if (rp2 && ci2 && v2 && vals && cols && rec && split && nnz_rows && final2 && ybuf) {
        memcpy(rp2, rp, sizeof(int) * (size_t)m);
        for (size_t i = (size_t)m; i < (size_t)m + 1 + slack; i++) rp2[i] = nitems;
        memcpy(ci2, ci, sizeof(int) * (size_t)nnz);
        memcpy(v2, v, sizeof(double) * (size_t)nnz);
        double t1 = now_s();
        oracle_cvr_convert(T, m, nitems, rp2, ci2, v2, vals, cols, rec, split, nnz_rows, final2);
        double t2 = now_s();
        double *yy = ybuf + slack; /* y[-1] is written by the reference's step-0 records */
        oracle_cvr_spmv(T, m, nitems, vals, cols, rec, split, nnz_rows, final2, x, yy);
        memcpy(y, yy, sizeof(double) * (size_t)m);
        double t3 = now_s();
        for (int it = 0; it < iters; it++) {
            memset(ybuf, 0, sizeof(double) * ((size_t)m + 2 * slack));
            oracle_cvr_spmv(T, m, nitems, vals, cols, rec, split, nnz_rows, final2, x, yy);
        }
        double t4 = now_s();
        if (convert_s) *convert_s = t2 - t1;
        if (exec_s) *exec_s = iters > 0 ? (t4 - t3) / iters : 0.0;
        rc = 0;
    }
    free(rp2); free(ci2); free(v2); free(vals); free(cols); free(rec); free(split);
    free(nnz_rows); free(final2); free(ybuf);
    return rc;
}
