// Support kernels: CSR validation, the augmented row pointer, the deterministic carry fixup
// shared by the CVR and CSR5 forms, and the plain-CSR kernel (baseline and in-GPU checker).

#include <cub/cub.cuh>

#include "pava_internal.h"

namespace pava {

namespace {

// Counts violations: row_ptr[0] != 0, row_ptr decreasing, row_ptr[m] != nnz, column outside
// [0, n).  The reference performs no such check (its loader trusts the file).
__global__ void validate_kernel(const int *__restrict__ rp, const int *__restrict__ ci, int m,
                                int n, int nnz, int *__restrict__ err) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    int bad = 0;
    for (long long r = tid; r < m; r += stride)
        if (rp[r + 1] < rp[r]) ++bad;
    if (tid == 0 && (rp[0] != 0 || rp[m] != nnz)) ++bad;
    if (bad == 0)  // only scan columns against a sane row pointer
        for (long long j = tid; j < nnz; j += stride) {
            const int c = ci[j];
            if (c < 0 || c >= n) ++bad;
        }
    if (bad) atomicAdd(err, bad);
}

struct EmptyRow {
    const int *rp;
    __host__ __device__ int operator()(int r) const { return rp[r + 1] == rp[r] ? 1 : 0; }
};

// arp[r] = rp[r] + (empty rows before r), r in [0, m]; arp[m+1] is set by the caller.
__global__ void arp_kernel(const int *__restrict__ rp, const int *__restrict__ empties, int m,
                           int *__restrict__ arp) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r <= m) arp[r] = rp[r] + empties[r];
}

__global__ void set_int_kernel(int *p, long long v) { *p = (int)v; }

// One warp per chunk c1.  A row R that spans chunks c0 < c1 (it starts in c0 and ends in c1)
// gets y[R] = carry_tail[c0] + sum(carry_head[c0+1 .. c1]); chunks in between lie entirely
// inside R and hold their whole contribution in carry_head.  The sum runs in a fixed order
// (lane-strided partial sums, then a fixed butterfly), so y is the same on every call.
__global__ void carry_fixup_kernel(const char *__restrict__ meta, size_t stride,
                                   const int *__restrict__ arp, long long L,
                                   const double *__restrict__ carry_head,
                                   const double *__restrict__ carry_tail, double *__restrict__ y,
                                   long long nchunks, int m) {
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long c1 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c1 < nchunks;
         c1 += nwarps) {
        const ChunkHdr *H = reinterpret_cast<const ChunkHdr *>(meta + c1 * stride);
        const unsigned sh = H->shared;
        if (!(sh & 1u)) continue;
        if ((sh & 2u) && H->nrows == 1) continue;  // R runs through c1 and beyond
        const int R = H->r_first;
        if (R >= m) continue;
        const long long c0 = (long long)arp[R] / L;
        double p = 0.0;
        for (long long j = c0 + 1 + lane; j <= c1; j += 32) p += carry_head[j];
        p = warp_sum(p);
        if (lane == 0) y[R] = carry_tail[c0] + p;
    }
}

// Plain CSR, V lanes per row, FP64: sum over the row in lane-strided order, then a fixed
// butterfly over the V lanes.
template <int V>
__global__ void __launch_bounds__(256)
csr_vector_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                  const double *__restrict__ v, const double *__restrict__ x,
                  double *__restrict__ y, int m) {
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = gt / V;
    const int sub = (int)(gt % V);
    const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
    double s = 0.0;
    if (row < m) {
        const int a = rp[row], b = rp[row + 1];
        for (int j = a + sub; j < b; j += V) {
            double val;
            int col;
            asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;"
                         : "=d"(val) : "l"(v + j), "l"(pf));
            asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
                         : "=r"(col) : "l"(ci + j), "l"(pf));
            s = fma(val, ld_x(x + col, pl), s);
        }
    }
#pragma unroll
    for (int d = V / 2; d > 0; d >>= 1) s += __shfl_xor_sync(FULL, s, d);
    if (row < m && sub == 0) y[row] = s;
}

}  // namespace

cudaError_t launch_validate(const int *rp, const int *ci, int m, int n, int nnz, int *d_err,
                            cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    long long work = (long long)(m > nnz ? m : nnz);
    long long blocks = (work + 255) / 256;
    if (blocks < 1) blocks = 1;
    if (blocks > 65535) blocks = 65535;
    validate_kernel<<<(unsigned)blocks, 256, 0, s>>>(rp, ci, m, n, nnz, d_err);
    return cudaGetLastError();
}

cudaError_t build_augmented_rowptr(const int *rp, int m, long long padded_total, int *arp,
                                   int *d_nempty, cudaStream_t s) {
    // empties[r] = number of empty rows before r (exclusive scan of the empty-row flags)
    int *empties = nullptr;
    cudaError_t e = cudaMallocAsync(&empties, sizeof(int) * ((size_t)m + 1), s);
    if (e != cudaSuccess) return e;
    cub::CountingInputIterator<int> rows(0);
    cub::TransformInputIterator<int, EmptyRow, cub::CountingInputIterator<int>> flags(
        rows, EmptyRow{rp});
    // empties[0] = 0, empties[1..m] = inclusive scan of flag(0..m-1)
    size_t tmp_bytes = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, flags, empties + 1, m, s);
    void *tmp = nullptr;
    e = cudaMallocAsync(&tmp, tmp_bytes > 0 ? tmp_bytes : 1, s);
    if (e != cudaSuccess) { cudaFreeAsync(empties, s); return e; }
    cudaMemsetAsync(empties, 0, sizeof(int), s);
    if (m > 0) cub::DeviceScan::InclusiveSum(tmp, tmp_bytes, flags, empties + 1, m, s);
    arp_kernel<<<(unsigned)(((long long)m + 1 + 255) / 256), 256, 0, s>>>(rp, empties, m, arp);
    set_int_kernel<<<1, 1, 0, s>>>(arp + m + 1, padded_total);
    cudaMemcpyAsync(d_nempty, empties + m, sizeof(int), cudaMemcpyDeviceToDevice, s);
    cudaFreeAsync(tmp, s);
    cudaFreeAsync(empties, s);
    return cudaGetLastError();
}

cudaError_t carry_fixup(const Handle &h, void *y, cudaStream_t s) {
    if (h.nchunks <= 0) return cudaSuccess;
    long long blocks = (h.nchunks * 32 + 255) / 256;
    const long long cap = (long long)h.sm_count * 16;
    if (blocks > cap) blocks = cap;
    carry_fixup_kernel<<<(unsigned)blocks, 256, 0, s>>>((const char *)h.meta, h.meta_stride,
                                                        h.arp, h.L, h.carry_head, h.carry_tail,
                                                        (double *)y, h.nchunks, h.m);
    return cudaGetLastError();
}

cudaError_t csr_spmv(const Handle &h, const void *x, void *y, cudaStream_t s) {
    if (h.m <= 0) return cudaSuccess;
    const long long threads = (long long)h.m * h.lanes_per_row;
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    const double *xd = (const double *)x;
    double *yd = (double *)y;
    switch (h.lanes_per_row) {
        case 1: csr_vector_kernel<1><<<blocks, 256, 0, s>>>(h.rp, h.ci, h.v, xd, yd, h.m); break;
        case 2: csr_vector_kernel<2><<<blocks, 256, 0, s>>>(h.rp, h.ci, h.v, xd, yd, h.m); break;
        case 4: csr_vector_kernel<4><<<blocks, 256, 0, s>>>(h.rp, h.ci, h.v, xd, yd, h.m); break;
        case 8: csr_vector_kernel<8><<<blocks, 256, 0, s>>>(h.rp, h.ci, h.v, xd, yd, h.m); break;
        case 16: csr_vector_kernel<16><<<blocks, 256, 0, s>>>(h.rp, h.ci, h.v, xd, yd, h.m); break;
        case 32: csr_vector_kernel<32><<<blocks, 256, 0, s>>>(h.rp, h.ci, h.v, xd, yd, h.m); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace pava
