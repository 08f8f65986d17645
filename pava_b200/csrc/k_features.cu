// Structural features of a CSR matrix, computed on the device, for the learned form selector.
//
// One warp per row (grid-stride).  Every statistic is accumulated in 64-bit integers (block
// partials, then one atomic per block), so the features are the same bits on every run.
// Columns are assumed sorted within a row (the engine's generators and .mtx path produce
// them so); the x-line count below is then the number of distinct 128-byte lines of an FP64
// x the row touches.
//
// Features (all floats):
//   0  log10(m)                          6  share of nonzeros in rows longer than 64
//   1  log10(nnz)                        7  share of rows with 1..4 nonzeros
//   2  log10(mean row length)            8  log10(mean |col - row| / n + 1e-7)
//   3  std / mean of row length          9  share of nonzeros with |col - row| <= 64
//   4  log10(max / mean row length)     10  distinct 128-byte x lines per nonzero
//   5  share of empty rows              11  log10(mean row span / n + 1e-7)

#include <math.h>

#include "pava_internal.h"

namespace pava {

namespace {

enum {
    S_LEN2,      // sum len^2
    S_EMPTY,     // empty rows
    S_LONGNNZ,   // nnz in rows longer than 64
    S_SHORT,     // rows with 1..4 nonzeros
    S_ABSDIST,   // sum |col - row|
    S_NEAR,      // nonzeros with |col - row| <= 64
    S_LINES,     // distinct x lines summed over rows
    S_SPAN,      // sum over non-empty rows of last col - first col + 1
    S_MAXLEN,    // max row length
    NSTAT
};

__global__ void __launch_bounds__(256)
features_kernel(const int *__restrict__ rp, const int *__restrict__ ci, int m,
                unsigned long long *__restrict__ stat) {
    __shared__ unsigned long long part[NSTAT];
    if (threadIdx.x < NSTAT) part[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned long long loc[NSTAT] = {0};
    for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m;
         r += warps) {
        const int a = rp[r], b = rp[r + 1];
        const long long len = b - a;
        unsigned long long dist = 0, near = 0, lines = 0;
        for (int j = a + lane; j < b; j += 32) {
            const int c = ci[j];
            const long long d = c >= r ? (long long)c - r : r - (long long)c;
            dist += (unsigned long long)d;
            near += d <= 64;
            lines += (j == a) || ((ci[j - 1] >> 4) != (c >> 4));
        }
        if (lane == 0) {
            loc[S_LEN2] += (unsigned long long)(len * len);
            loc[S_EMPTY] += len == 0;
            loc[S_LONGNNZ] += len > 64 ? (unsigned long long)len : 0ull;
            loc[S_SHORT] += len >= 1 && len <= 4;
            if (len > 0) loc[S_SPAN] += (unsigned long long)(ci[b - 1] - ci[a] + 1);
            if ((unsigned long long)len > loc[S_MAXLEN]) loc[S_MAXLEN] = (unsigned long long)len;
        }
        loc[S_ABSDIST] += dist;
        loc[S_NEAR] += near;
        loc[S_LINES] += lines;
    }
    for (int k = 0; k < NSTAT; ++k) {
        if (k == S_MAXLEN) atomicMax(&part[k], loc[k]);
        else if (loc[k]) atomicAdd(&part[k], loc[k]);
    }
    __syncthreads();
    if (threadIdx.x < NSTAT) {
        if (threadIdx.x == S_MAXLEN) atomicMax(&stat[S_MAXLEN], part[S_MAXLEN]);
        else if (part[threadIdx.x]) atomicAdd(&stat[threadIdx.x], part[threadIdx.x]);
    }
}

}  // namespace

cudaError_t matrix_features(const int *rp, const int *ci, int m, int n, int nnz, float *out,
                            cudaStream_t s) {
    unsigned long long *d = nullptr;
    cudaError_t e = cudaMallocAsync(&d, sizeof(unsigned long long) * NSTAT, s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(d, 0, sizeof(unsigned long long) * NSTAT, s);
    unsigned long long h[NSTAT] = {0};
    if (e == cudaSuccess && m > 0) {
        long long blocks = ((long long)m * 32 + 255) / 256;
        if (blocks > 4096) blocks = 4096;
        features_kernel<<<(unsigned)blocks, 256, 0, s>>>(rp, ci, m, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(d, s);
    if (e != cudaSuccess) return e;
    const double M = m > 0 ? m : 1, Z = nnz > 0 ? nnz : 1, N = n > 0 ? n : 1;
    const double mean = nnz / M;
    const double var = (double)h[S_LEN2] / M - mean * mean;
    const double nonempty = M - (double)h[S_EMPTY];
    out[0] = (float)log10(M);
    out[1] = (float)log10(Z);
    out[2] = (float)log10(mean > 1e-9 ? mean : 1e-9);
    out[3] = (float)(mean > 0 ? sqrt(var > 0 ? var : 0) / mean : 0);
    out[4] = (float)log10(mean > 0 && h[S_MAXLEN] > 0 ? (double)h[S_MAXLEN] / mean : 1.0);
    out[5] = (float)((double)h[S_EMPTY] / M);
    out[6] = (float)((double)h[S_LONGNNZ] / Z);
    out[7] = (float)((double)h[S_SHORT] / M);
    out[8] = (float)log10((double)h[S_ABSDIST] / Z / N + 1e-7);
    out[9] = (float)((double)h[S_NEAR] / Z);
    out[10] = (float)((double)h[S_LINES] / Z);
    out[11] = (float)log10((nonempty > 0 ? (double)h[S_SPAN] / nonempty : 0.0) / N + 1e-7);
    return cudaSuccess;
}

}  // namespace pava

extern "C" pava_status pava_features(const pava_csr *A, float *out12, void *stream) {
    using namespace pava;
    if (!A || !out12) { set_last_error("NULL argument"); return PAVA_E_INVALID_ARG; }
    if (!A->on_device) { set_last_error("pava_features needs a device CSR"); return PAVA_E_INVALID_ARG; }
    if (A->m < 0 || A->nnz < 0) { set_last_error("negative size"); return PAVA_E_INVALID_ARG; }
    cudaError_t e = matrix_features(A->row_ptr, A->col_idx, A->m, A->n, A->nnz, out12,
                                    (cudaStream_t)stream);
    if (e != cudaSuccess) {
        set_last_error(std::string("features: ") + cudaGetErrorString(e));
        return PAVA_E_CUDA;
    }
    return PAVA_SUCCESS;
}
