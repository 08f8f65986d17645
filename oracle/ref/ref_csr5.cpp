/*
 * Test infrastructure (oracle only).  Compiles the reference's CSR5 engine
 * (csr5/anonymouslib_avx512.h and csr5/detail/avx512/*.h) from the reference tree and exposes
 * it as plain C functions for the parity tests and the timed CPU baseline.  Nothing in the
 * product links this file.
 *
 * It drives anonymouslibHandle (csr5/anonymouslib_avx512.h:14-276) the way conduct_csr5
 * (csr5/csr5.h:72-179) does -- inputCSR, setX, setSigma(12), asCSR5, spmv -- but not through
 * conduct_csr5/runKernel, which fall off the end of non-void functions.  The handle transposes
 * the column/value arrays it is given in place (csr5/detail/avx512/format_avx512.h:428), so
 * it is given copies.  Only the first spmv after asCSR5, into zeroed y, is returned: the
 * per-thread calibrator is cleared only in asCSR5 (csr5/anonymouslib_avx512.h:152) and
 * accumulates on every later call (csr5/detail/avx512/csr5_spmv_avx512.h:41,277).
 */
#include <omp.h>
#include <string.h>
#include <stdlib.h>
#include <sys/time.h>

#define private public /* the oracle reads the handle's tile arrays to pin the port */
#include "csr5/anonymouslib_avx512.h"
#undef private

static double wall_s() {
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + tv.tv_usec / 1e6;
}

template <class T> static T *zalloc(size_t n) {
    T *p = (T *)_mm_malloc(sizeof(T) * (n ? n : 1), 64);
    if (p) memset(p, 0, sizeof(T) * (n ? n : 1));
    return p;
}

extern "C" {

/* Tile parameters the reference derives for sigma (csr5/anonymouslib_avx512.h:124-139), for
 * sizing the optional outputs of pava_ref_csr5: out[0]=p, out[1]=bit_y_offset,
 * out[2]=bit_scansum_offset, out[3]=num_packet. */
void pava_ref_csr5_params(int nnz, int sigma, int *out) {
    int omega = ANONYMOUSLIB_CSR5_OMEGA;
    int base = 2, bit_y = 1, bit_s = 1;
    while (base < omega * sigma) { base *= 2; bit_y++; }
    base = 2;
    while (base < omega) { base *= 2; bit_s++; }
    int bit_all = bit_y + bit_s + sigma;
    out[0] = (int)ceil((double)nnz / (double)(omega * sigma));
    out[1] = bit_y;
    out[2] = bit_s;
    out[3] = (int)ceil((double)bit_all / 32.0);
}

/* Converts CSR -> CSR5 with the reference (sigma given, omega = 8), runs one SpMV into zeroed
 * y (the oracle output, m entries), then `iters` timed SpMV calls into a scratch vector.
 * The CSR given here is used as is (callers pad nnz as they wish).  Optional outputs (NULL to
 * skip): tile_ptr (p+1), tile_desc (p*8*num_packet), desc_offset_ptr (p+1), desc_offset
 * (up to desc_offset_cap), num_offsets, the transposed cols/vals (nnz each).  Returns the
 * reference status (0 = ANONYMOUSLIB_SUCCESS) or -100 on allocation failure. */
int pava_ref_csr5(int nthreads, int sigma, int m, int n, int nnz, const int *rp, const int *ci,
                  const double *v, const double *x, double *y, int iters, double *convert_s,
                  double *exec_s, unsigned *out_tile_ptr, unsigned *out_tile_desc,
                  int *out_desc_offset_ptr, int *out_desc_offset, int desc_offset_cap,
                  int *out_num_offsets, int *out_cols, double *out_vals) {
    omp_set_num_threads(nthreads);
    const size_t slack = 256;
    int *rp2 = zalloc<int>((size_t)m + 1 + slack);
    int *ci2 = zalloc<int>((size_t)nnz + slack);
    double *v2 = zalloc<double>((size_t)nnz + slack);
    double *x2 = zalloc<double>((size_t)n + slack);
    double *yout = zalloc<double>((size_t)m + slack);
    double *yit = zalloc<double>((size_t)m + slack);
    if (!rp2 || !ci2 || !v2 || !x2 || !yout || !yit) return -100;
    memcpy(rp2, rp, sizeof(int) * ((size_t)m + 1));
    memcpy(ci2, ci, sizeof(int) * (size_t)nnz);
    memcpy(v2, v, sizeof(double) * (size_t)nnz);
    memcpy(x2, x, sizeof(double) * (size_t)n);

    anonymouslibHandle<int, unsigned int, double> A(m, n);
    int err = A.inputCSR(nnz, rp2, ci2, v2);
    if (err == 0) err = A.setX(x2);
    A.setSigma(sigma);
    double t1 = wall_s();
    if (err == 0) err = A.asCSR5();
    double t2 = wall_s();
    double t3 = t2, t4 = t2;
    if (err == 0) {
        if (out_tile_ptr) memcpy(out_tile_ptr, A._csr5_partition_pointer, sizeof(unsigned) * ((size_t)A._p + 1));
        if (out_tile_desc)
            memcpy(out_tile_desc, A._csr5_partition_descriptor,
                   sizeof(unsigned) * (size_t)A._p * ANONYMOUSLIB_CSR5_OMEGA * A._num_packet);
        if (out_desc_offset_ptr)
            memcpy(out_desc_offset_ptr, A._csr5_partition_descriptor_offset_pointer, sizeof(int) * ((size_t)A._p + 1));
        if (out_num_offsets) *out_num_offsets = A._num_offsets;
        if (out_desc_offset && A._num_offsets) {
            int k = A._num_offsets < desc_offset_cap ? A._num_offsets : desc_offset_cap;
            memcpy(out_desc_offset, A._csr5_partition_descriptor_offset, sizeof(int) * (size_t)k);
        }
        if (out_cols) memcpy(out_cols, ci2, sizeof(int) * (size_t)nnz);
        if (out_vals) memcpy(out_vals, v2, sizeof(double) * (size_t)nnz);
        err = A.spmv(1.0, yout);
        memcpy(y, yout, sizeof(double) * (size_t)m);
        t3 = wall_s();
        for (int i = 0; i < iters && err == 0; i++) err = A.spmv(1.0, yit);
        t4 = wall_s();
        A.asCSR();
    }
    if (convert_s) *convert_s = t2 - t1;
    if (exec_s) *exec_s = iters > 0 ? (t4 - t3) / iters : 0.0;
    _mm_free(rp2); _mm_free(ci2); _mm_free(v2); _mm_free(x2); _mm_free(yout); _mm_free(yit);
    return err;
}

} /* extern "C" */
