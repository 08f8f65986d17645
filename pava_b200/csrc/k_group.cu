// CSR row-group kernel: SpMV and multi-RHS SpMM (Y = A X, X row-major n x k) on plain CSR,
// FP64 or FP32-compensated, for short-row and batched matrices.
//
// A group of GL lanes (a power of two <= 32) owns one row at a time.  Inside the group, KC
// lanes span the k right-hand sides (lane c holds columns c, c + KC, ..., KPL of them) and
// ES = GL / KC element slices split the row's nonzeros (slice e takes elements e, e + ES, ...).
// For k = 1 this is the vector-CSR kernel with GL lanes per row; for k = 32, GL = KC = 32 it is
// one warp per row reading 256-byte rows of X.  A slice's partial sums are combined over the
// ES slices with a fixed xor butterfly, so every call gives the same bits.
//
// The launch is persistent: the grid is sized to the resident capacity of the GPU and warps
// take tiles of TR consecutive rows in grid-stride order (tile t to warp t mod warps), which
// keeps one launch per SpMV/SpMM whatever the number of rows -- the batched path (a
// block-diagonal union of many small matrices) relies on this.

#include "k_stream.cuh"
#include "pava_internal.h"

namespace pava {

namespace {

__device__ __forceinline__ double ld_val(const double *p, uint64_t pol) {
    double r;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;"
                 : "=d"(r) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ float ld_val(const float *p, uint64_t pol) {
    float r;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
                 : "=f"(r) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ int ld_col(const int *p, uint64_t pol) {
    int r;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
                 : "=r"(r) : "l"(p), "l"(pol));
    return r;
}

constexpr int GROUP_THREADS = 256;
// resident blocks per SM: more warps in flight for the narrow shapes
template <int KPL> constexpr int group_minb() { return KPL == 1 ? 6 : (KPL == 2 ? 5 : 4); }
// elements in flight per lane
template <int KPL> constexpr int group_unroll() { return KPL == 1 ? 4 : (KPL == 2 ? 2 : 1); }

template <int KPL, typename VT>
__global__ void __launch_bounds__(GROUP_THREADS, group_minb<KPL>())
csr_group_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                 const VT *__restrict__ v, const VT *__restrict__ X, long long ldx,
                 double *__restrict__ Y, long long ldy, int m, int k, int gl_shift,
                 int kc_shift, int tile_rows) {
    constexpr int U = group_unroll<KPL>();
    const int lane = threadIdx.x & 31;
    const int gl = 1 << gl_shift, kc = 1 << kc_shift;
    const int grp = lane >> gl_shift;          // group within the warp
    const int gpw = 32 >> gl_shift;            // groups (rows in flight) per warp
    const int gi = lane & (gl - 1);
    const int e = gi >> kc_shift;              // element slice
    const int es = gl >> kc_shift;             // slices per row
    const int cl = gi & (kc - 1);              // first column of this lane
    const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
    const long long ntiles = ((long long)m + tile_rows - 1) / tile_rows;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int rounds = tile_rows / gpw;        // rows per group per tile

    bool colok[KPL];
#pragma unroll
    for (int p = 0; p < KPL; ++p) colok[p] = cl + p * kc < k;

    for (long long t = (((long long)blockIdx.x * blockDim.x) + threadIdx.x) >> 5; t < ntiles;
         t += nwarps) {
        for (int i = 0; i < rounds; ++i) {
            const long long r = t * tile_rows + (long long)i * gpw + grp;
            const bool valid = r < m;
            int a = 0, b = 0;
            if (valid) {
                a = rp[r];
                b = rp[r + 1];
            }
            Acc<VT> acc[KPL];
            int j = a + e;
            // U elements at a time: all value and column loads first, then all gathers, so
            // U memory round trips overlap instead of running one after another
            for (; j + (U - 1) * es < b; j += U * es) {
                VT val[U];
                int col[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    val[u] = ld_val(v + j + u * es, pf);
                    col[u] = ld_col(ci + j + u * es, pf);
                }
                VT xv[U][KPL];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const VT *xr = X + (long long)col[u] * ldx + cl;
#pragma unroll
                    for (int p = 0; p < KPL; ++p) xv[u][p] = colok[p] ? ld_x(xr + p * kc, pl) : VT(0);
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int p = 0; p < KPL; ++p)
                        if (colok[p]) acc[p].add(val[u], xv[u][p]);
            }
            for (; j < b; j += es) {
                const VT val = ld_val(v + j, pf);
                const VT *xr = X + (long long)ld_col(ci + j, pf) * ldx + cl;
#pragma unroll
                for (int p = 0; p < KPL; ++p)
                    if (colok[p]) acc[p].add(val, ld_x(xr + p * kc, pl));
            }
#pragma unroll
            for (int p = 0; p < KPL; ++p) {
                double s = acc[p].value();
                for (int o = kc; o < gl; o <<= 1) s += __shfl_xor_sync(FULL, s, o);
                if (valid && e == 0 && colok[p]) Y[r * ldy + cl + p * kc] = s;
            }
        }
    }
}

int ilog2(int v) {
    int s = 0;
    while ((1 << s) < v) ++s;
    return s;
}

template <typename VT>
cudaError_t launch_group(const Handle &h, const void *X, long long ldx, void *Y, long long ldy,
                         int k, cudaStream_t s) {
    const int gl = h.lanes_per_row, kc = h.col_lanes, kpl = h.cols_per_lane;
    const int gpw = 32 / gl;
    const int tr = h.rows_per_tile;
    const long long ntiles = ((long long)h.m + tr - 1) / tr;
    const long long want = (ntiles + (GROUP_THREADS / 32) - 1) / (GROUP_THREADS / 32);
    const int minb = kpl == 1 ? group_minb<1>() : (kpl == 2 ? group_minb<2>() : group_minb<4>());
    const long long cap = (long long)h.sm_count * minb;
    const unsigned grid = (unsigned)(want < cap ? (want > 0 ? want : 1) : cap);
    (void)gpw;
    const int gs = ilog2(gl), ks = ilog2(kc);
    const VT *x = (const VT *)X;
    const VT *v = (const VT *)h.v;
    double *y = (double *)Y;
    switch (kpl) {
        case 1:
            csr_group_kernel<1, VT><<<grid, GROUP_THREADS, 0, s>>>(h.rp, h.ci, v, x, ldx, y, ldy,
                                                                 h.m, k, gs, ks, tr);
            break;
        case 2:
            csr_group_kernel<2, VT><<<grid, GROUP_THREADS, 0, s>>>(h.rp, h.ci, v, x, ldx, y, ldy,
                                                                 h.m, k, gs, ks, tr);
            break;
        case 4:
            csr_group_kernel<4, VT><<<grid, GROUP_THREADS, 0, s>>>(h.rp, h.ci, v, x, ldx, y, ldy,
                                                                 h.m, k, gs, ks, tr);
            break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

__global__ void narrow_kernel(const double *__restrict__ src, float *__restrict__ dst,
                              long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        dst[i] = (float)src[i];
}

}  // namespace

cudaError_t csr_spmm(const Handle &h, const void *X, long long ldx, void *Y, long long ldy,
                     int k, cudaStream_t s) {
    if (h.m <= 0 || k <= 0) return cudaSuccess;
    if (h.precision == PAVA_PREC_FP32C) return launch_group<float>(h, X, ldx, Y, ldy, k, s);
    return launch_group<double>(h, X, ldx, Y, ldy, k, s);
}

cudaError_t csr_spmv(const Handle &h, const void *x, void *y, cudaStream_t s) {
    return csr_spmm(h, x, 1, y, 1, 1, s);
}

cudaError_t narrow_to_float(const double *src, float *dst, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    long long blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    narrow_kernel<<<(unsigned)blocks, 256, 0, s>>>(src, dst, n);
    return cudaGetLastError();
}

}  // namespace pava
