/*
 * ORACLE -- test infrastructure only (never linked by the product).
 *
 * Scalar restatement of the reference CSR5 engine for omega = 8 lanes (csr5/): the conversion
 * steps of asCSR5 (csr5/anonymouslib_avx512.h:107-221; csr5/detail/avx512/format_avx512.h) and
 * the SpMV csr5_spmv (csr5/detail/avx512/csr5_spmv_avx512.h:346-382) with its compute,
 * calibrate and tail kernels.  The 8-lane vector steps are written lane by lane with the same
 * operation order as the AVX-512 code (the masked blends, the lane rotation, hscan_avx512 of
 * csr5/detail/avx512/utils_avx512.h:65-90 and GCC's _mm512_reduce_add_pd tree), so the tile
 * arrays match bit for bit and y matches to the last bit on the matrices the tests use.
 *
 * One input difference is fixed here: generate_partition_pointer_s2_kernel reads
 * row_ptr[m+1] for the last tile (format_avx512.h:43-51), one past the caller's array; this
 * restatement reads it as 0, which is what the oracle's reference build supplies (zeroed
 * slack).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include "oracle.h"

#define OMEGA 8

void oracle_csr5_params(int nnz, int sigma, oracle_csr5_info *info) {
    int base = 2, bit_y = 1, bit_s = 1;
    while (base < OMEGA * sigma) { base *= 2; bit_y++; }
    base = 2;
    while (base < OMEGA) { base *= 2; bit_s++; }
    int bit_all = bit_y + bit_s + sigma;
    info->sigma = sigma;
    info->omega = OMEGA;
    info->bit_y_offset = bit_y;
    info->bit_scansum_offset = bit_s;
    info->num_packet = (int)ceil((double)bit_all / 32.0);
    info->p = (int)ceil((double)nnz / (double)(OMEGA * sigma));
    info->num_offsets = 0;
    info->tail_partition_start = 0;
}

/* binary_search_right_boundary_kernel, csr5/detail/avx512/utils_avx512.h:23-45 */
static int bsearch_right(const int *d, int key, int size) {
    int start = 0, stop = size - 1, med;
    while (stop >= start) {
        med = (stop + start) / 2;
        if (key >= d[med]) start = med + 1; else stop = med - 1;
    }
    return start;
}

/* scan_single, csr5/detail/avx512/utils_avx512.h:49-62 (exclusive scan) */
static void scan_single(int *s, int l) {
    int old_val = s[0], new_val;
    s[0] = 0;
    for (int i = 1; i < l; i++) {
        new_val = s[i];
        s[i] = old_val + s[i - 1];
        old_val = new_val;
    }
}

static inline int rp_at(const int *rp, int m, int i) { return i <= m ? rp[i] : 0; }

int oracle_csr5_convert(int m, int nnz, const int *rp, const int *cols, const double *vals,
                        const oracle_csr5_info *info, unsigned *tile_ptr, unsigned *tile_desc,
                        int *desc_off_ptr, int *tcols, double *tvals) {
    const int sigma = info->sigma, p = info->p, np = info->num_packet;
    const int bit_y = info->bit_y_offset, bit_s = info->bit_scansum_offset;
    const int bit_all = bit_y + bit_s;
    /* generate_partition_pointer s1 (format_avx512.h:8-28) */
    for (int gid = 0; gid <= p; gid++) {
        int boundary = gid * sigma * OMEGA;
        boundary = boundary > nnz ? nnz : boundary;
        tile_ptr[gid] = (unsigned)(bsearch_right(rp, boundary, m + 1) - 1);
    }
    /* s2: flag tiles that contain an empty row (format_avx512.h:30-64) */
    for (int gid = 0; gid < p; gid++) {
        unsigned start = (tile_ptr[gid] << 1) >> 1, stop = (tile_ptr[gid + 1] << 1) >> 1;
        if (start == stop) continue;
        int dirty = 0;
        for (int r = (int)start; r <= (int)stop; r++)
            if (rp_at(rp, m, r) == rp_at(rp, m, r + 1)) { dirty = 1; break; }
        if (dirty) tile_ptr[gid] = start | 0x80000000u;
    }
    /* descriptor s1: row-start bits (format_avx512.h:85-121) */
    for (int par = 0; par < p - 1; par++) {
        int r0 = (int)(tile_ptr[par] & 0x7FFFFFFF), r1 = (int)(tile_ptr[par + 1] & 0x7FFFFFFF);
        for (int rid = r0; rid <= r1; rid++) {
            int ptr = rp[rid];
            int pid = ptr / (OMEGA * sigma);
            if (pid == par) {
                int lx = (ptr / sigma) % OMEGA;
                int glid = ptr % sigma + bit_all;
                int ly = glid / 32, llid = glid % 32;
                tile_desc[pid * OMEGA * np + ly * OMEGA + lx] |= 0x1u << (31 - llid);
            }
        }
    }
    /* descriptor s2: y_offset and scansum_offset per lane (format_avx512.h:123-233) */
    for (int par = 0; par < p - 1; par++) {
        int segn_scan[OMEGA + 1] = {0};
        int present_arr[OMEGA + 1] = {0};
        present_arr[OMEGA] = 1;
        int with_empty = (int)((tile_ptr[par] >> 31) & 0x1);
        unsigned r0 = tile_ptr[par] & 0x7FFFFFFF, r1 = tile_ptr[par + 1] & 0x7FFFFFFF;
        if (r0 == r1) continue;
        for (int lane = 0; lane < OMEGA; lane++) {
            int start = 0, stop = 0, segn, present = 0, ly = 0;
            present |= !lane;
            unsigned first_packet = tile_desc[par * OMEGA * np + lane];
            unsigned bitflag = (first_packet << bit_all) | ((unsigned)present << 31);
            start = !((bitflag >> 31) & 0x1);
            present |= (bitflag >> 31) & 0x1;
            for (int i = 1; i < sigma; i++) {
                if ((!ly && i == 32 - bit_all) || (ly && (i - (32 - bit_all)) % 32 == 0)) {
                    ly++;
                    bitflag = tile_desc[par * OMEGA * np + ly * OMEGA + lane];
                }
                int norm_i = !ly ? i : i - (32 - bit_all);
                stop += (bitflag >> (31 - norm_i % 32)) & 0x1;
                present |= (bitflag >> (31 - norm_i % 32)) & 0x1;
            }
            segn = stop - start + present;
            segn = segn > 0 ? segn : 0;
            segn_scan[lane] = segn;
            present_arr[lane] = present;
        }
        scan_single(segn_scan, OMEGA + 1);
        if (with_empty) {
            desc_off_ptr[par] = segn_scan[OMEGA];
            desc_off_ptr[p] += segn_scan[OMEGA];
        }
        for (int lane = 0; lane < OMEGA; lane++) {
            int y_offset = segn_scan[lane], scansum_offset = 0, next1 = lane + 1;
            if (present_arr[lane])
                while (!present_arr[next1] && next1 < OMEGA) { scansum_offset++; next1++; }
            unsigned fp = tile_desc[par * OMEGA * np + lane];
            y_offset = lane ? y_offset - 1 : 0;
            fp |= (unsigned)y_offset << (32 - bit_y);
            fp |= (unsigned)scansum_offset << (32 - bit_all);
            tile_desc[par * OMEGA * np + lane] = fp;
        }
    }
    if (desc_off_ptr[p]) scan_single(desc_off_ptr, p + 1);
    /* aosoa_transpose R2C, out of place (format_avx512.h:365-450) */
    memcpy(tcols, cols, sizeof(int) * (size_t)nnz);
    memcpy(tvals, vals, sizeof(double) * (size_t)nnz);
    for (int par = 0; par < p - 1; par++) {
        if (tile_ptr[par] == tile_ptr[par + 1]) continue;
        const int base = par * OMEGA * sigma;
        for (int idx = 0; idx < OMEGA * sigma; idx++) {
            int iy = idx % sigma, ix = idx / sigma;
            tcols[base + iy * OMEGA + ix] = cols[base + idx];
            tvals[base + iy * OMEGA + ix] = vals[base + idx];
        }
    }
    return desc_off_ptr[p];
}

void oracle_csr5_offsets(const int *rp, const oracle_csr5_info *info, const unsigned *tile_ptr,
                         const unsigned *tile_desc, const int *desc_off_ptr, int *desc_off) {
    const int sigma = info->sigma, p = info->p, np = info->num_packet;
    const int bit_y = info->bit_y_offset, bit_all = info->bit_y_offset + info->bit_scansum_offset;
    const int bit_bitflag = 32 - bit_all;
    /* generate_partition_descriptor_offset_kernel, format_avx512.h:271-343 */
    for (int par = 0; par < p - 1; par++) {
        if (!((tile_ptr[par] >> 31) & 0x1)) continue;
        int r0 = (int)(tile_ptr[par] & 0x7FFFFFFF), r1 = (int)(tile_ptr[par + 1] & 0x7FFFFFFF);
        int off = desc_off_ptr[par];
        for (int lane = 0; lane < OMEGA; lane++) {
            int ly = 0;
            unsigned d = tile_desc[par * OMEGA * np + lane];
            int y_offset = (int)(d >> (32 - bit_y));
            d = d << bit_all;
            d = lane ? d : (d | 0x80000000u);
            int local_bit = (d >> 31) & 0x1;
            if (local_bit && lane) {
                int idx = par * OMEGA * sigma + lane * sigma;
                desc_off[off + y_offset] = bsearch_right(&rp[r0 + 1], idx, r1 - r0) - 1;
                y_offset++;
            }
            for (int i = 1; i < sigma; i++) {
                if ((!ly && i == bit_bitflag) || (ly && !(31 & (i - bit_bitflag)))) {
                    ly++;
                    d = tile_desc[par * OMEGA * np + ly * OMEGA + lane];
                }
                int norm_i = 31 & (!ly ? i : i - bit_bitflag);
                local_bit = (d >> (31 - norm_i)) & 0x1;
                if (local_bit) {
                    int idx = par * OMEGA * sigma + lane * sigma + i;
                    desc_off[off + y_offset] = bsearch_right(&rp[r0 + 1], idx, r1 - r0) - 1;
                    y_offset++;
                }
            }
        }
    }
}

/* GCC's _mm512_reduce_add_pd order: ((a4+a0)+(a6+a2)) + ((a5+a1)+(a7+a3)). */
static inline double reduce8(const double *a) {
    double t0 = a[4] + a[0], t1 = a[5] + a[1], t2 = a[6] + a[2], t3 = a[7] + a[3];
    return (t2 + t0) + (t3 + t1);
}

/* hscan_avx512 (utils_avx512.h:65-90): inclusive scan as three shifted adds. */
static inline void hscan8(double *s) {
    double a[8], b[8];
    for (int k = 0; k < 8; k++) a[k] = s[k] + (k >= 1 ? s[k - 1] : 0.0);
    for (int k = 0; k < 8; k++) b[k] = a[k] + (k >= 2 ? a[k - 2] : 0.0);
    for (int k = 0; k < 8; k++) s[k] = b[k] + (k >= 4 ? b[k - 4] : 0.0);
}

void oracle_csr5_spmv(int T, int m, const int *rp, const int *ocols, const double *ovals,
                      const int *tcols, const double *tvals, const oracle_csr5_info *info,
                      const unsigned *tile_ptr, const unsigned *tile_desc,
                      const int *desc_off_ptr, const int *desc_off, const double *x, double *y) {
    const int sigma = info->sigma, p = info->p, np = info->num_packet;
    const int bit_y = info->bit_y_offset, bit_s = info->bit_scansum_offset;
    const int chunk = (int)ceil((double)(p - 1) / (double)T);
    const int active = chunk > 0 ? (int)ceil((p - 1.0) / chunk) : 0;
    double *cal = (double *)calloc((size_t)T, sizeof(double));
    /* spmv_csr5_compute_kernel, csr5_spmv_avx512.h:52-289 */
    for (int tid = 0; tid < T && chunk > 0; tid++) {
        int start_row_start = tid < active ? (int)(tile_ptr[tid * chunk] & 0x7FFFFFFF) : 0;
        int p0 = tid * chunk, p1 = (tid + 1) * chunk;
        if (p1 > p - 1) p1 = p - 1;
        for (int par = p0; par < p1; par++) {
            const double *vp = tvals + (size_t)par * OMEGA * sigma;
            const int *cp = tcols + (size_t)par * OMEGA * sigma;
            unsigned row_start = tile_ptr[par];
            const unsigned row_stop = tile_ptr[par + 1] & 0x7FFFFFFF;
            if (row_start == row_stop) { /* partition_fast_track, :8-49 */
                int direct = (tile_desc[par * OMEGA * np] >> (31 - (bit_y + bit_s))) & 0x1;
                double acc[8] = {0};
                for (int i = 0; i < sigma; i++)
                    for (int l = 0; l < 8; l++)
                        acc[l] = fma(vp[i * OMEGA + l], x[cp[i * OMEGA + l]], acc[l]);
                double sum = reduce8(acc);
                if ((int)row_start == start_row_start && !direct) cal[tid] += sum;
                else if (direct) y[row_start] = sum;
                else y[row_start] += sum;
                continue;
            }
            const int empty_rows = (row_start >> 31) & 0x1;
            row_start &= 0x7FFFFFFF;
            double *y_local = y + row_start + 1;
            const int offp = empty_rows ? desc_off_ptr[par] : 0;
            unsigned yoff[8], so[8], dd[8];
            int bit[8], direct[8], start[8], stop[8];
            double sum[8], first_sum[8], last_sum[8], tmp[8];
            for (int l = 0; l < 8; l++) {
                unsigned d = tile_desc[par * OMEGA * np + l];
                yoff[l] = d >> (32 - bit_y);
                so[l] = (d << bit_y) >> (32 - bit_s);
                dd[l] = d << (bit_y + bit_s);
                bit[l] = (int)(dd[l] >> 31);
                first_sum[l] = 0.0;
                stop[l] = 0;
            }
            const int first_direct = bit[0];
            const int first_all_direct = (par == tid * chunk) ? first_direct : 0;
            bit[0] = 1;
            for (int l = 0; l < 8; l++) {
                start[l] = bit[l] ? 0 : 1;
                direct[l] = (l == 0) ? 0 : bit[l];
                sum[l] = vp[l] * x[cp[l]];
            }
            for (int i = 1; i < sigma; i++) {
                int any = 0;
                for (int l = 0; l < 8; l++) {
                    bit[l] = (int)((dd[l] >> (31 - i)) & 0x1);
                    any |= bit[l];
                }
                if (any) {
                    for (int l = 0; l < 8; l++) {
                        if (direct[l] && bit[l]) {
                            int yi = empty_rows ? desc_off[offp + (int)yoff[l]] : (int)yoff[l];
                            y_local[yi] = sum[l];
                            yoff[l]++;
                        }
                    }
                    for (int l = 0; l < 8; l++) {
                        if (!direct[l] && bit[l]) first_sum[l] = sum[l];
                        if (bit[l]) sum[l] = 0.0;
                        direct[l] |= bit[l];
                        if (direct[l]) stop[l] += 1;
                    }
                }
                for (int l = 0; l < 8; l++)
                    sum[l] = fma(vp[i * OMEGA + l], x[cp[i * OMEGA + l]], sum[l]);
            }
            for (int l = 0; l < 8; l++) {
                first_sum[l] = direct[l] ? first_sum[l] : sum[l];
                last_sum[l] = sum[l];
            }
            double s8[8];
            for (int k = 0; k < 7; k++) s8[k] = (start[k + 1] == 1) ? first_sum[k + 1] : 0.0;
            s8[7] = 0.0;
            for (int k = 0; k < 8; k++) tmp[k] = s8[k];
            hscan8(s8);
            double shifted[8];
            for (int k = 0; k < 8; k++) shifted[k] = s8[k + (int)so[k]];
            for (int k = 0; k < 8; k++) {
                double r = (shifted[k] - s8[k]) + tmp[k];
                last_sum[k] = last_sum[k] + ((start[k] <= stop[k]) ? r : 0.0);
            }
            for (int l = 0; l < 8; l++) {
                if (direct[l]) {
                    int yi = empty_rows ? desc_off[offp + (int)yoff[l]] : (int)yoff[l];
                    y_local[yi] = last_sum[l];
                }
            }
            double s0 = direct[0] ? first_sum[0] : last_sum[0];
            s0 = s0 + 0.0; /* _mm512_mask_reduce_add_pd of one lane */
            if ((int)row_start == start_row_start && !first_all_direct) cal[tid] += s0;
            else if (first_direct) y[row_start] = s0;
            else y[row_start] += s0;
        }
    }
    /* spmv_csr5_calibrate_kernel, :292-308 */
    int ncali = active < T ? active : T;
    for (int i = 0; i < ncali; i++) y[tile_ptr[i * chunk] & 0x7FFFFFFF] += cal[i];
    /* spmv_csr5_tail_partition_kernel, :311-342; the reference build keeps this sum unfused
     * (multiply then add), unlike the intrinsic FMAs of the tile kernel */
    const int tps = info->tail_partition_start;
    const int first_tail = (p - 1) * OMEGA * sigma;
    for (int row = tps; row < m; row++) {
        int i0 = row == tps ? first_tail : rp[row];
        int i1 = rp[row + 1];
        double s = 0.0;
        for (int idx = i0; idx < i1; idx++) s += ovals[idx] * x[ocols[idx]];
        if (row == tps && rp[row] != first_tail) y[row] = y[row] + s;
        else y[row] = s;
    }
    free(cal);
}

static double now_s(void) {
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + tv.tv_usec / 1e6;
}

int oracle_csr5_run(int T, int sigma, int m, int n, int nnz, const int *rp, const int *ci,
                    const double *v, const double *x, double *y, double *convert_s,
                    double *exec_s, int iters) {
    (void)n;
    oracle_csr5_info info;
    oracle_csr5_params(nnz, sigma, &info);
    const int p = info.p;
    unsigned *tp = (unsigned *)calloc((size_t)p + 2, sizeof(unsigned));
    unsigned *td = (unsigned *)calloc((size_t)p * OMEGA * info.num_packet + 8, sizeof(unsigned));
    int *dop = (int *)calloc((size_t)p + 2, sizeof(int));
    int *tc = (int *)calloc((size_t)nnz + 8, sizeof(int));
    double *tv = (double *)calloc((size_t)nnz + 8, sizeof(double));
    double *yb = (double *)calloc((size_t)m + 8, sizeof(double));
    int *dof = NULL;
    int rc = -1;
    if (tp && td && dop && tc && tv && yb) {
        double t1 = now_s();
        int noff = oracle_csr5_convert(m, nnz, rp, ci, v, &info, tp, td, dop, tc, tv);
        info.num_offsets = noff;
        info.tail_partition_start = (int)((tp[p - 1] << 1) >> 1);
        if (noff) {
            dof = (int *)calloc((size_t)noff + 8, sizeof(int));
            if (dof) oracle_csr5_offsets(rp, &info, tp, td, dop, dof);
        }
        double t2 = now_s();
        if (!noff || dof) {
            oracle_csr5_spmv(T, m, rp, ci, v, tc, tv, &info, tp, td, dop, dof, x, y);
            double t3 = now_s();
            for (int it = 0; it < iters; it++) {
                memset(yb, 0, sizeof(double) * (size_t)m);
                oracle_csr5_spmv(T, m, rp, ci, v, tc, tv, &info, tp, td, dop, dof, x, yb);
            }
            double t4 = now_s();
            if (convert_s) *convert_s = t2 - t1;
            if (exec_s) *exec_s = iters > 0 ? (t4 - t3) / iters : 0.0;
            rc = 0;
        }
    }
    free(tp); free(td); free(dop); free(tc); free(tv); free(yb); free(dof);
    return rc;
}
