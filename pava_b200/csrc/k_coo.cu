// COO -> sorted CSR on the device: the GPU form of the loader's conversion (readCOOMatrix's
// symmetric expansion and 1-based shift, utils/basicMatrix.cpp:63-253, and convertCOO2CSR,
// :350-415, which calls MKL's mkl_dcsrcoo there).
//
// Entries are keyed (row << 32 | column) and sorted by a stable LSD radix sort (cub), so rows
// and the columns inside a row come out ascending and duplicates stay as separate entries in
// input order -- the same result as the host conversion, pava_coo_to_csr.  With `symmetric`,
// every off-diagonal entry (r, c) also yields (c, r), as a symmetric Matrix Market file
// stores one triangle.  The row pointer is then read off the sorted keys: element j writes
// rp[r] = j for every row r in (row[j-1], row[j]].

#include <string.h>

#include <cub/cub.cuh>

#include "pava_internal.h"

namespace pava {

namespace {

unsigned grid_of(long long work) {
    long long b = (work + 255) / 256;
    if (b < 1) b = 1;
    if (b > 16384) b = 16384;
    return (unsigned)b;
}

// flag[k] = 1 for an off-diagonal entry when mirroring; counts indices out of range.
__global__ void coo_flags_kernel(const int *__restrict__ rows, const int *__restrict__ cols,
                                 long long nnz, int base, int m, int n, int symmetric,
                                 int *__restrict__ flag, int *__restrict__ bad) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    int nb = 0;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) {
        const int r = rows[k] - base, c = cols[k] - base;
        const bool ok = r >= 0 && r < m && c >= 0 && c < n && (!symmetric || (c < m && r < n));
        nb += !ok;
        flag[k] = (ok && symmetric && r != c) ? 1 : 0;
    }
    if (nb) atomicAdd(bad, nb);
}

__global__ void coo_keys_kernel(const int *__restrict__ rows, const int *__restrict__ cols,
                                const double *__restrict__ vals, long long nnz, int base,
                                const int *__restrict__ mirror_pos, int symmetric,
                                unsigned long long *__restrict__ keys, double *__restrict__ v) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) {
        const unsigned long long r = (unsigned)(rows[k] - base), c = (unsigned)(cols[k] - base);
        keys[k] = (r << 32) | c;
        v[k] = vals[k];
        if (symmetric && r != c) {
            const long long q = nnz + mirror_pos[k];
            keys[q] = (c << 32) | r;
            v[q] = vals[k];
        }
    }
}

// Row pointer and columns from the sorted keys; j = total stands for a virtual element of
// row m, which closes every remaining row.
__global__ void coo_rowptr_kernel(const unsigned long long *__restrict__ keys, long long total,
                                  int m, int *__restrict__ rp, int *__restrict__ ci) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j <= total; j += stride) {
        const long long row = j < total ? (long long)(keys[j] >> 32) : m;
        const long long prev = j > 0 ? (long long)(keys[j - 1] >> 32) : -1;
        for (long long r = prev + 1; r <= row; ++r) rp[r] = (int)j;
        if (j < total) ci[j] = (int)(keys[j] & 0xffffffffull);
    }
}

int key_bits(int m) {
    int b = 0;
    while ((1ll << b) < (long long)m + 1) ++b;
    return 32 + b;
}

}  // namespace

}  // namespace pava

extern "C" pava_status pava_coo_to_csr_device(int m, int n, long long nnz, const int *rows,
                                              const int *cols, const double *vals,
                                              int index_base, int symmetric, void *stream,
                                              pava_csr *out) {
    using namespace pava;
    if (!out) { set_last_error("out is NULL"); return PAVA_E_INVALID_ARG; }
    memset(out, 0, sizeof(*out));
    if (m < 0 || n < 0 || nnz < 0 || (nnz > 0 && (!rows || !cols || !vals)) ||
        (index_base != 0 && index_base != 1)) {
        set_last_error("bad sizes, NULL arrays or index base other than 0 / 1");
        return PAVA_E_INVALID_ARG;
    }
    if (nnz > 2147483000LL) { set_last_error("more than 2^31 entries"); return PAVA_E_TOO_LARGE; }
    cudaStream_t s = (cudaStream_t)stream;
    int *flag = nullptr, *mpos = nullptr, *d_bad = nullptr, *rp = nullptr, *ci = nullptr;
    unsigned long long *keys = nullptr, *keys2 = nullptr;
    double *v = nullptr, *v2 = nullptr;
    void *tmp = nullptr;
    auto cleanup = [&]() {
        cudaFree(flag); cudaFree(mpos); cudaFree(d_bad); cudaFree(keys); cudaFree(keys2);
        cudaFree(v); cudaFree(tmp);
    };
    auto fail_e = [&](cudaError_t e) {
        cleanup();
        cudaFree(rp); cudaFree(ci); cudaFree(v2);
        set_last_error(std::string("COO -> CSR: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PAVA_E_NOMEM : PAVA_E_CUDA;
    };
    const size_t nz = (size_t)(nnz ? nnz : 1);
    cudaError_t e = cudaMalloc(&flag, sizeof(int) * nz);
    if (e == cudaSuccess) e = cudaMalloc(&mpos, sizeof(int) * nz);
    if (e == cudaSuccess) e = cudaMalloc(&d_bad, sizeof(int) * 2);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, sizeof(int) * 2, s);
    if (e == cudaSuccess && nnz > 0) {
        coo_flags_kernel<<<grid_of(nnz), 256, 0, s>>>(rows, cols, nnz, index_base, m, n,
                                                      symmetric, flag, d_bad);
        e = cudaGetLastError();
    }
    size_t tb = 0;
    if (e == cudaSuccess && nnz > 0) e = cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, mpos, (int)nnz, s);
    if (e == cudaSuccess && nnz > 0) e = cudaMalloc(&tmp, tb ? tb : 1);
    if (e == cudaSuccess && nnz > 0) e = cub::DeviceScan::ExclusiveSum(tmp, tb, flag, mpos, (int)nnz, s);
    if (e == cudaSuccess && nnz > 0)  // mirrored count = mpos[last] + flag[last]
        e = cub::DeviceReduce::Sum(nullptr, tb, flag, d_bad + 1, (int)nnz, s);
    cudaFree(tmp);
    tmp = nullptr;
    if (e == cudaSuccess && nnz > 0) e = cudaMalloc(&tmp, tb ? tb : 1);
    if (e == cudaSuccess && nnz > 0) e = cub::DeviceReduce::Sum(tmp, tb, flag, d_bad + 1, (int)nnz, s);
    int h[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_bad, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail_e(e);
    if (h[0]) {
        cleanup();
        set_last_error("COO -> CSR: " + std::to_string(h[0]) + " entries outside the matrix");
        return PAVA_E_INVALID_CSR;
    }
    const long long total = nnz + h[1];
    if (total > 2147483000LL) {
        cleanup();
        set_last_error("more than 2^31 entries after the symmetric expansion");
        return PAVA_E_TOO_LARGE;
    }
    const size_t tz = (size_t)(total ? total : 1);
    e = cudaMalloc(&keys, sizeof(unsigned long long) * tz);
    if (e == cudaSuccess) e = cudaMalloc(&keys2, sizeof(unsigned long long) * tz);
    if (e == cudaSuccess) e = cudaMalloc(&v, sizeof(double) * tz);
    if (e == cudaSuccess) e = cudaMalloc(&v2, sizeof(double) * tz);
    if (e == cudaSuccess) e = cudaMalloc(&rp, sizeof(int) * ((size_t)m + 1));
    if (e == cudaSuccess) e = cudaMalloc(&ci, sizeof(int) * tz);
    if (e == cudaSuccess && nnz > 0) {
        coo_keys_kernel<<<grid_of(nnz), 256, 0, s>>>(rows, cols, vals, nnz, index_base, mpos,
                                                     symmetric, keys, v);
        e = cudaGetLastError();
    }
    cudaFree(tmp);
    tmp = nullptr;
    if (e == cudaSuccess && total > 0)
        e = cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, v, v2, (int)total, 0,
                                            key_bits(m), s);
    if (e == cudaSuccess && total > 0) e = cudaMalloc(&tmp, tb ? tb : 1);
    if (e == cudaSuccess && total > 0)
        e = cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, v, v2, (int)total, 0,
                                            key_bits(m), s);
    if (e == cudaSuccess) {
        coo_rowptr_kernel<<<grid_of(total + 1), 256, 0, s>>>(keys2, total, m, rp, ci);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail_e(e);
    cleanup();
    out->m = m;
    out->n = n;
    out->nnz = (int)total;
    out->row_ptr = rp;
    out->col_idx = ci;
    out->vals = v2;
    out->on_device = 1;
    return PAVA_SUCCESS;
}
