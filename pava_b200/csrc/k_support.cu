// Support kernels: CSR validation, the augmented row pointer and the deterministic carry fixup
// shared by the CVR and CSR5 forms.

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

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
                                   long long nchunks, int m, unsigned long long *err) {
    // launched as a programmatic dependent of the SpMV kernel: wait until that grid has
    // finished and its carries are visible (returns at once for an ordinary launch)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long c1 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c1 < nchunks;
         c1 += nwarps) {
        const ChunkHdr *H = reinterpret_cast<const ChunkHdr *>(meta + c1 * stride);
        const unsigned sh = H->shared;
        if (!(sh & 1u)) continue;
        if ((sh & 2u) && H->nrows == 1) continue;  // R runs through c1 and beyond
        const int R = H->r_first;
        if (R >= m || !guard(err, R >= 0, G_Y, R)) continue;
        const long long c0 = (long long)arp[R] / L;
        if (!guard(err, c0 >= 0 && c0 <= c1, G_CARRY, c0)) continue;
        double p = 0.0;
        for (long long j = c0 + 1 + lane; j <= c1; j += 32) p += carry_head[j];
        p = warp_sum(p);
        if (lane == 0) y[R] = carry_tail[c0] + p;
    }
}

// Warp per chunk.  Chunk c holds the augmented elements [c*L, (c+1)*L); augmentation only
// inserts zero elements, so its nonzeros are the CSR's positions [p0, p1).  base = midpoint of
// their smallest and largest column: 16-bit offsets then reach any chunk whose columns span
// at most 65,534 (a chunk without nonzeros gets 0).
__global__ void chunk_colbase_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                                     const int *__restrict__ arp, int m, long long nchunks,
                                     long long L, int *__restrict__ colbase) {
    const int lane = threadIdx.x & 31;
    const long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= nchunks) return;  // warp-uniform
    const long long s = c * L, e = s + L;
    const int nr = m + 2;
    // CSR position of augmented element `at`, clamped to row r's nonzeros
    auto pos = [&](int r, long long at) -> long long {
        if (r >= m) return rp[m];
        const long long len = rp[r + 1] - rp[r];
        long long off = at - arp[r];
        off = off < 0 ? 0 : (off > len ? len : off);
        return rp[r] + off;
    };
    const long long p0 = pos(upper_bound_m1(arp, nr, s), s);
    const long long p1 = pos(upper_bound_m1(arp, nr, e - 1), e);
    int mn = 0x7fffffff, mx = -1;
    for (long long p = p0 + lane; p < p1; p += 32) {
        const int col = ci[p];
        mn = col < mn ? col : mn;
        mx = col > mx ? col : mx;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int a = __shfl_xor_sync(FULL, mn, o), b = __shfl_xor_sync(FULL, mx, o);
        mn = a < mn ? a : mn;
        mx = b > mx ? b : mx;
    }
    if (lane == 0) colbase[c] = mx >= 0 ? (int)(((long long)mn + mx) / 2) : 0;
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

cudaError_t chunk_colbase(const Handle &h, const int *rp, const int *ci, cudaStream_t s) {
    if (h.nchunks <= 0) return cudaSuccess;
    chunk_colbase_kernel<<<(unsigned)((h.nchunks * 32 + 255) / 256), 256, 0, s>>>(
        rp, ci, h.arp, h.m, h.nchunks, h.L, h.colbase);
    return cudaGetLastError();
}

cudaError_t build_augmented_rowptr(const int *rp, int m, long long padded_total, int *arp,
                                   int *d_nempty, cudaStream_t s) {
    // empties[r] = number of empty rows before r (exclusive scan of the empty-row flags)
    int *empties = nullptr;
    cudaError_t e = cudaMallocAsync(&empties, sizeof(int) * ((size_t)m + 1), s);
    if (e != cudaSuccess) return e;
    auto flags = thrust::make_transform_iterator(thrust::make_counting_iterator(0), EmptyRow{rp});
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
    // programmatic dependent launch: the fixup grid is launched while the SpMV grid runs (its
    // launch latency hidden) and waits for it in griddepcontrol.wait
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, carry_fixup_kernel, (const char *)h.meta, h.meta_stride,
                              (const int *)h.arp, h.L, (const double *)h.carry_head,
                              (const double *)h.carry_tail, (double *)y, h.nchunks, h.m,
                              guard_word());
}

}  // namespace pava
