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
#ifndef PAVA_SELL_MINB
#define PAVA_SELL_MINB 3
#endif

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

template <bool B> struct SFlag { static constexpr bool value = B; };

// SpMV: one warp per slice (grid-stride over slices, persistent grid).  The slice's blocks run
// through a register pipeline -- values two blocks ahead, columns three, x one -- and each lane
// accumulates its own row; the slice ends with one coalesced store of 32 rows.
template <typename VT, typename IT>
__global__ void __launch_bounds__(SELL_WARPS * 32, PAVA_SELL_MINB)
sell_spmv_kernel(const SellSlice *__restrict__ meta, const VT *__restrict__ vals,
                 const IT *__restrict__ cols, const VT *__restrict__ x,
                 double *__restrict__ y, long long nslices, int m, int n,
                 unsigned long long *err) {
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
        Acc<VT> acc;
        // CHK: the slice pads some rows, so each gather tests its column
        auto walk = [&](auto chk_tag) {
            constexpr bool CHK = decltype(chk_tag)::value;
            auto gather4 = [&](const CBlk<IT> &cbk, VT (&xs)[4]) {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    xs[q] = CHK ? cbk.gather(q, xb, pl, xlo, xhi, err)
                                : cbk.gather_all(q, xb, pl, xlo, xhi, err);
            };
            CBlk<IT> c1 = CBlk<IT>::load(cb, NB > 1 ? 1 : 0, lane, pf);
            CBlk<IT> c2 = CBlk<IT>::load(cb, NB > 2 ? 2 : 0, lane, pf);
            VBlk<VT> v0 = VBlk<VT>::load(vb, 0, lane, pf);
            VBlk<VT> v1 = VBlk<VT>::load(vb, NB > 1 ? 1 : 0, lane, pf);
            VT x0[4];
            {
                const CBlk<IT> c0 = CBlk<IT>::load(cb, 0, lane, pf);
                gather4(c0, x0);
            }
#pragma unroll 1
            for (int blk = 0; blk < NB; ++blk) {
                CBlk<IT> cn = c2;
                VBlk<VT> vn = v1;
                if (blk + 3 < NB) cn = CBlk<IT>::load(cb, blk + 3, lane, pf);
                if (blk + 2 < NB) vn = VBlk<VT>::load(vb, blk + 2, lane, pf);
                VT x1[4];
                if (blk + 1 < NB) gather4(c1, x1);
#pragma unroll
                for (int q = 0; q < 4; ++q) acc.add(v0.get(q), x0[q]);
                c1 = c2; c2 = cn;
                v0 = v1; v1 = vn;
#pragma unroll
                for (int q = 0; q < 4; ++q) x0[q] = x1[q];
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
    const long long cap = (long long)h.sm_count * PAVA_SELL_MINB;
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
