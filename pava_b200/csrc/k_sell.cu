// Sliced ELLPACK (SELL): conversion and SpMV for sm_100a.
//
// A slice is 32 consecutive rows, one per lane of a warp.  Each slice stores its rows padded to
// the length of its longest row (rounded up to 4), in the 4-step block layout of k_stream.cuh:
// element i of the slice's lane k (row 32 s + k) sits at off_s + vals_offset(i, k), so at step
// i the 32 lanes read one 16-byte vector each per stream and gather x for the i-th nonzero of
// 32 consecutive rows.  On matrices whose neighbouring rows have the same pattern (stencils,
// banded and block structures) those 32 gathers land on one or two 128-byte lines, where the
// CVR and CSR5 walks (a lane runs through consecutive nonzeros of a few rows) spread them over
// many lines.  Every row is summed by one lane from its first to its last nonzero, so there
// are no row-start flags, no cross-lane combine and no carries: one pass, one coalesced y
// store per slice, no fixup launch.  Padding elements (value 0, no column) read no x.
//
// The price is the padding, so the form is for matrices whose rows in a slice have similar
// lengths; pava_create refuses it (PAVA_E_UNSUPPORTED_PARAMS) when padding would more than
// double the stored elements.  No counterpart in the reference (pava's engines are CVR and
// CSR5); it is a third engine form beside them, offered by the autotuner and the selector.

#include <cub/cub.cuh>

#include "k_stream.cuh"
#include "pava_internal.h"

namespace pava {

namespace {

constexpr int SELL_WARPS = 8;

template <typename IT> __device__ __forceinline__ IT sell_enc(int col, int base, int *ovf);
template <> __device__ __forceinline__ int sell_enc<int>(int col, int, int *) { return col; }
template <> __device__ __forceinline__ short sell_enc<short>(int col, int base, int *ovf) {
    if (col < 0) return DELTA_NONE;
    const int d = col - base;
    if (d < -32767 || d > 32767) { atomicOr(ovf, 1); return DELTA_NONE; }
    return (short)d;
}

// Warp per slice: the slice's blocks of 4 steps (its longest row, rounded up), whether any lane
// pads, and (for 16-bit offsets) the base column, the middle of the slice's column range.
__global__ void sell_plan_kernel(const int *__restrict__ rp, const int *__restrict__ ci, int m,
                                 long long nslices, int want_base, SellSlice *__restrict__ meta,
                                 int *__restrict__ nblk_out) {
    const int lane = threadIdx.x & 31;
    const long long s = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= nslices) return;  // warp-uniform
    const long long r = s * 32 + lane;
    const int a = r < m ? rp[r] : 0, len = r < m ? rp[r + 1] - a : 0;
    int mx = len;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int t = __shfl_xor_sync(FULL, mx, o);
        mx = t > mx ? t : mx;
    }
    const int nblk = (mx + 3) / 4;
    const bool pads = __any_sync(FULL, len < 4 * nblk);
    int cmin = 0x7fffffff, cmax = -1;
    if (want_base) {
        for (int j = 0; j < len; ++j) {
            const int c = ci[a + j];
            cmin = c < cmin ? c : cmin;
            cmax = c > cmax ? c : cmax;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int u = __shfl_xor_sync(FULL, cmin, o), w = __shfl_xor_sync(FULL, cmax, o);
            cmin = u < cmin ? u : cmin;
            cmax = w > cmax ? w : cmax;
        }
    }
    if (lane == 0) {
        meta[s].off = 0;
        meta[s].nblk = nblk;
        meta[s].colbase = cmax >= 0 ? (int)(((long long)cmin + cmax) / 2) : 0;
        meta[s].flags = pads ? 1u : 0u;
        nblk_out[s] = nblk;
    }
}

// Warp per slice: lane k copies row 32 s + k into the slice's block layout, padding with
// (0, no column).  blk_off[s] = the slice's first block (exclusive scan of nblk).
template <typename VT, typename IT>
__global__ void sell_fill_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                                 const double *__restrict__ v, int m, long long nslices,
                                 const int *__restrict__ blk_off, SellSlice *__restrict__ meta,
                                 VT *__restrict__ vals, IT *__restrict__ cols, int *ovf) {
    const int lane = threadIdx.x & 31;
    const long long s = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= nslices) return;
    const long long off = (long long)blk_off[s] * 128;
    const int nblk = meta[s].nblk, base = meta[s].colbase;
    const long long r = s * 32 + lane;
    const int a = r < m ? rp[r] : 0, len = r < m ? rp[r + 1] - a : 0;
    for (int i = 0; i < 4 * nblk; ++i) {
        const bool in = i < len;
        vals[off + vals_offset<VT>(i, lane)] = in ? (VT)v[a + i] : VT(0);
        cols[off + cols_offset(i, lane)] = sell_enc<IT>(in ? ci[a + i] : -1, base, ovf);
    }
    if (lane == 0) meta[s].off = (int)off;
}

// Pipeline depth (blocks of 4 steps the value and column loads run ahead of their use) and
// resident CTAs per SM of each value form.
#ifndef PAVA_SELL_D64
#define PAVA_SELL_D64 2
#endif
#ifndef PAVA_SELL_D32
#define PAVA_SELL_D32 2
#endif
#ifndef PAVA_SELL_MINB64
#define PAVA_SELL_MINB64 3
#endif
#ifndef PAVA_SELL_MINB32
#define PAVA_SELL_MINB32 4
#endif

// Row sums.  FP64: FMA.  FP32 values and x: a product of two FP32 numbers is exact in FP64
// (24 + 24 significant bits < 53), so the FP32 form widens both factors and sums the exact
// products with FP64 FMAs -- an FP64 sum of exact terms, one rounding per nonzero.
template <typename VT> struct RowAcc;
template <> struct RowAcc<double> {
    double s = 0.0;
    __device__ __forceinline__ void add(double v, double x) { s = fma(v, x, s); }
    __device__ __forceinline__ double value() const { return s; }
    __device__ __forceinline__ void reset() { s = 0.0; }
};
template <> struct RowAcc<float> {
    double s = 0.0;
    __device__ __forceinline__ void add(float v, float x) { s = fma((double)v, (double)x, s); }
    __device__ __forceinline__ double value() const { return s; }
    __device__ __forceinline__ void reset() { s = 0.0; }
};

template <typename VT> struct SellShape;
template <> struct SellShape<double> {
    static constexpr int D = PAVA_SELL_D64, MINB = PAVA_SELL_MINB64;
};
template <> struct SellShape<float> {
    static constexpr int D = PAVA_SELL_D32, MINB = PAVA_SELL_MINB32;
};

template <bool B> struct SFlag { static constexpr bool value = B; };

// SpMV: one warp per slice (grid-stride over slices, persistent grid: the warps of the grid
// work on neighbouring slices at any time, so the streams are read close to in order).  The
// slice's blocks run through register rings of D slots: the values of block b + D and the
// columns of block b + D + 1 are loaded while block b is summed and the x of block b + 1 is
// gathered.  Each lane accumulates its own row; the slice ends with one coalesced store of 32
// rows.
template <typename VT, typename IT>
__global__ void __launch_bounds__(SELL_WARPS * 32, SellShape<VT>::MINB)
sell_spmv_kernel(const SellSlice *__restrict__ meta, const VT *__restrict__ vals,
                 const IT *__restrict__ cols, const VT *__restrict__ x,
                 double *__restrict__ y, long long nslices, int m, int n,
                 unsigned long long *err) {
    constexpr int D = SellShape<VT>::D;
    static_assert(D >= 2 && D % 2 == 0, "the x ring of two slots needs an even depth");
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
    const long long nwarps = (long long)gridDim.x * SELL_WARPS;
    for (long long s = (long long)blockIdx.x * SELL_WARPS + w; s < nslices; s += nwarps) {
        const SellSlice S = meta[s];
        const int NB = S.nblk;
        const VT *vb = vals + S.off;
        const IT *cb = cols + S.off;
        const int xbase = sizeof(IT) == 2 ? S.colbase : 0;  // base of the 16-bit offsets
        const VT *xb = x + xbase;
        const int xlo = -xbase, xhi = n - xbase;
        RowAcc<VT> acc;
        // CHK: the slice pads some rows, so each gather tests its column
        auto walk = [&](auto chk_tag) {
            constexpr bool CHK = decltype(chk_tag)::value;
            auto gather4 = [&](const CBlk<IT> &cbk, VT (&xs)[4]) {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    xs[q] = CHK ? cbk.gather(q, xb, pl, xlo, xhi, err)
                                : cbk.gather_all(q, xb, pl, xlo, xhi, err);
            };
            VBlk<VT> v[D];
            CBlk<IT> c[D];
            VT xs[2][4];
#pragma unroll
            for (int j = 0; j < D; ++j) {
                if (j < NB) {
                    v[j] = VBlk<VT>::load(vb, j, lane, pf);
                    c[j] = CBlk<IT>::load(cb, j, lane, pf);
                }
            }
            gather4(c[0], xs[0]);
            if (D < NB) c[0] = CBlk<IT>::load(cb, D, lane, pf);
#pragma unroll 1
            for (int b0 = 0; b0 < NB; b0 += D) {
#pragma unroll
                for (int j = 0; j < D; ++j) {  // block b = b0 + j sits in slot j
                    const int b = b0 + j;
                    if (b < NB) {
                        const int jn = (j + 1) % D;  // slot of block b + 1
                        if (b + 1 < NB) {
                            gather4(c[jn], xs[(j + 1) & 1]);
                            if (b + 1 + D < NB) c[jn] = CBlk<IT>::load(cb, b + 1 + D, lane, pf);
                        }
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc.add(v[j].get(q), xs[j & 1][q]);
                        if (b + D < NB) v[j] = VBlk<VT>::load(vb, b + D, lane, pf);
                    }
                }
            }
        };
        if (NB > 0) {
            if (S.flags & 1u) walk(SFlag<true>{});
            else walk(SFlag<false>{});
        }
        const long long r = s * 32 + lane;
        if (r < m) y[r] = acc.value();
    }
}

template <typename VT, typename IT>
cudaError_t fill_t(Handle &h, const int *rp, const int *ci, const double *v, const int *blk_off,
                   int *ovf, cudaStream_t s) {
    const long long threads = h.nchunks * 32;
    sell_fill_kernel<VT, IT><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(
        rp, ci, v, h.m, h.nchunks, blk_off, (SellSlice *)h.meta, (VT *)h.vals, (IT *)h.cols,
        ovf);
    return cudaGetLastError();
}

template <typename VT, typename IT>
cudaError_t spmv_t(const Handle &h, const void *x, void *y, cudaStream_t s) {
    const long long want = (h.nchunks + SELL_WARPS - 1) / SELL_WARPS;
    const long long cap = (long long)h.sm_count * SellShape<VT>::MINB;
    const unsigned grid = (unsigned)(want < cap ? want : cap);
    sell_spmv_kernel<VT, IT><<<grid, SELL_WARPS * 32, 0, s>>>(
        (const SellSlice *)h.meta, (const VT *)h.vals, (const IT *)h.cols, (const VT *)x,
        (double *)y, h.nchunks, h.m, h.n, guard_word());
    return cudaGetLastError();
}

}  // namespace

cudaError_t sell_plan(Handle &h, const int *rp, const int *ci, int *d_blk_off, int *d_total_blk,
                      cudaStream_t s) {
    const long long ns = h.nchunks;
    const long long threads = ns * 32;
    int *nblk = nullptr;
    cudaError_t e = cudaMallocAsync(&nblk, sizeof(int) * (size_t)(ns + 1), s);
    if (e != cudaSuccess) return e;
    sell_plan_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(
        rp, ci, h.m, ns, h.index_mode == PAVA_INDEX_DELTA16 ? 1 : 0, (SellSlice *)h.meta, nblk);
    e = cudaGetLastError();
    // blk_off[0..ns] = exclusive scan of nblk (blk_off[ns] = total blocks)
    if (e == cudaSuccess) e = cudaMemsetAsync(nblk + ns, 0, sizeof(int), s);
    size_t tmp_bytes = 0;
    if (e == cudaSuccess)
        e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, nblk, d_blk_off, (int)(ns + 1), s);
    void *tmp = nullptr;
    if (e == cudaSuccess) e = cudaMallocAsync(&tmp, tmp_bytes ? tmp_bytes : 1, s);
    if (e == cudaSuccess)
        e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, nblk, d_blk_off, (int)(ns + 1), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_total_blk, d_blk_off + ns, sizeof(int), cudaMemcpyDeviceToDevice, s);
    if (tmp) cudaFreeAsync(tmp, s);
    cudaFreeAsync(nblk, s);
    return e;
}

cudaError_t sell_fill(Handle &h, const int *rp, const int *ci, const double *v,
                      const int *d_blk_off, int *ovf, cudaStream_t s) {
    if (h.nchunks <= 0) return cudaSuccess;
    const bool f32 = h.precision == PAVA_PREC_FP32C, d16 = h.index_mode == PAVA_INDEX_DELTA16;
    if (!f32 && !d16) return fill_t<double, int>(h, rp, ci, v, d_blk_off, ovf, s);
    if (!f32 && d16) return fill_t<double, short>(h, rp, ci, v, d_blk_off, ovf, s);
    if (f32 && !d16) return fill_t<float, int>(h, rp, ci, v, d_blk_off, ovf, s);
    return fill_t<float, short>(h, rp, ci, v, d_blk_off, ovf, s);
}

cudaError_t sell_spmv(const Handle &h, const void *x, void *y, cudaStream_t s) {
    if (h.nchunks <= 0) return cudaSuccess;
    const bool f32 = h.precision == PAVA_PREC_FP32C, d16 = h.index_mode == PAVA_INDEX_DELTA16;
    if (!f32 && !d16) return spmv_t<double, int>(h, x, y, s);
    if (!f32 && d16) return spmv_t<double, short>(h, x, y, s);
    if (f32 && !d16) return spmv_t<float, int>(h, x, y, s);
    return spmv_t<float, short>(h, x, y, s);
}

}  // namespace pava
