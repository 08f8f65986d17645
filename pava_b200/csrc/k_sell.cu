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
// The SpMV stages the value and column streams through shared memory with bulk asynchronous
// copies (cp.async.bulk, completion counted on an mbarrier): a warp keeps two pieces of its
// slices in flight in its own shared-memory stages while it sums a third from shared memory,
// so the bytes in flight per SM are set by shared memory (~200 KB), not by registers.
//
// The price is the padding, so the form is for matrices whose rows in a slice have similar
// lengths; pava_create refuses it (PAVA_E_UNSUPPORTED_PARAMS) when padding would more than
// double the stored elements.  No counterpart in the reference (pava's engines are CVR and
// CSR5); it is a third engine form beside them, offered by the autotuner and the selector.

#include <atomic>
#include <climits>

#include <cub/cub.cuh>

#include "k_bulk.cuh"
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
    int mn = len;  // the shortest row: blocks before mn / 4 hold no padding
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int t = __shfl_xor_sync(FULL, mn, o);
        mn = t < mn ? t : mn;
    }
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
        meta[s].flags = pads ? 1u | ((unsigned)(mn / 4) << 1) : 0u;
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

// Bulk-copy staging.  A stage holds one piece: up to KB consecutive blocks of one slice
// (KB = the blocks of about 3 KB of value and column stream); each warp owns STAGES stages and
// an mbarrier per stage; CTAS_PER_SM CTAs of SELL_WARPS warps share an SM.
constexpr int STAGE_BYTES = 3072, STAGES = 2, CTAS_PER_SM = 4;
template <typename VT, typename IT> struct Stage {
    static constexpr int BPB = 128 * (int)(sizeof(VT) + sizeof(IT));  // bytes per block
    static constexpr int KB = STAGE_BYTES / BPB > 0 ? STAGE_BYTES / BPB : 1;
    static constexpr int VBYTES = KB * 128 * (int)sizeof(VT), CBYTES = KB * 128 * (int)sizeof(IT);
    static constexpr int WARP_BYTES = STAGES * (VBYTES + CBYTES) + 128;  // + barriers
    static constexpr int CTA_BYTES = SELL_WARPS * WARP_BYTES;
    static_assert(STAGES * 8 <= 128 && WARP_BYTES % 128 == 0, "stage layout");
};

// SpMV.  Warps take slices in turn (grid-stride: the warps of the grid work on neighbouring
// slices at any time, so the streams are read close to in order).  Each warp walks its slices
// as a sequence of pieces (<= KB blocks of one slice) with two cursors: the producer (lane 0
// issues the bulk copies of a piece into the next free stage) runs STAGES pieces ahead of the
// consumer, which waits for its stage's copies, sums the piece's blocks from shared memory
// -- gathering the x of block i + 1 while block i is summed -- and hands the stage back.  A
// slice's last piece stores its 32 rows; empty slices (no blocks) store zero rows.  A wait
// that gives up counts itself in wait_err[0] (the first slice in wait_err[1]); the warp then
// waits, again bounded, for the copies it still has in flight and stops.
template <typename VT, typename IT>
__global__ void __launch_bounds__(SELL_WARPS * 32, CTAS_PER_SM)
sell_spmv_kernel(const SellSlice *__restrict__ meta, const VT *__restrict__ vals,
                 const IT *__restrict__ cols, const VT *__restrict__ x,
                 double *__restrict__ y, long long nslices, int m, int n,
                 unsigned long long *err, unsigned long long *wait_err) {
    using ST = Stage<VT, IT>;
    constexpr int KB = ST::KB;
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned char *wbase = smem + w * ST::WARP_BYTES;  // [barriers | value stages | column stages]
    const unsigned bar0 = (unsigned)__cvta_generic_to_shared(wbase);
    const VT *sv = reinterpret_cast<const VT *>(wbase + 128);
    const IT *sc = reinterpret_cast<const IT *>(wbase + 128 + STAGES * ST::VBYTES);
    const unsigned sv0 = bar0 + 128, sc0 = bar0 + 128 + STAGES * ST::VBYTES;
    if (lane == 0) {
        for (int k = 0; k < STAGES; ++k) mbar_init(bar0 + 8 * k);
        mbar_init_fence();
    }
    __syncwarp();
    const uint64_t pl = policy_evict_last();
    const long long nwarps = (long long)gridDim.x * SELL_WARPS;
    const long long first = (long long)blockIdx.x * SELL_WARPS + w;

    // producer cursor: slice ps (with blocks), next block pb
    long long ps = first;
    int pb = 0;
    SellSlice pm{0, 0, 0, 0u};
    if (ps < nslices) pm = meta[ps];
    while (ps < nslices && pm.nblk == 0) {
        ps += nwarps;
        if (ps < nslices) pm = meta[ps];
    }
    auto issue = [&](int k) {
        const int len = min(KB, pm.nblk - pb);
        const long long e0 = (long long)pm.off + (long long)pb * 128;
        if (lane == 0) {
            const unsigned vb = (unsigned)(len * 128 * (int)sizeof(VT));
            const unsigned cb = (unsigned)(len * 128 * (int)sizeof(IT));
            proxy_fence();  // the stage's last reads come before the copy's writes
            mbar_expect_tx(bar0 + 8 * k, vb + cb);
            bulk_g2s(sv0 + k * ST::VBYTES, vals + e0, vb, bar0 + 8 * k);
            bulk_g2s(sc0 + k * ST::CBYTES, cols + e0, cb, bar0 + 8 * k);
        }
        pb += KB;
        if (pb >= pm.nblk) {
            pb = 0;
            do {
                ps += nwarps;
                if (ps < nslices) pm = meta[ps];
            } while (ps < nslices && pm.nblk == 0);
        }
    };
    int pending = 0;
#pragma unroll
    for (int k = 0; k < STAGES; ++k)
        if (ps < nslices) { issue(k); ++pending; }

    // consumer cursor: slice cs, next block cb; it writes the rows of empty slices
    long long cs = first;
    int cb = 0;
    SellSlice cm{0, 0, 0, 0u};
    auto skip_empty = [&]() {
        while (cs < nslices) {
            cm = meta[cs];
            if (cm.nblk > 0) break;
            const long long r = cs * 32 + lane;
            if (r < m) y[r] = 0.0;
            cs += nwarps;
        }
    };
    skip_empty();
    unsigned phases = 0;  // bit k: parity the consumer waits for on stage k
    int k = 0;
    RowAcc<VT> acc;
    while (cs < nslices) {
        if (!mbar_wait(bar0 + 8 * k, (phases >> k) & 1u)) {
            if (lane == 0) {
                atomicAdd(&wait_err[0], 1ull);
                atomicCAS(&wait_err[1], 0ull, (unsigned long long)cs + 1);
            }
            break;
        }
        phases ^= 1u << k;
        --pending;
        const int len = min(KB, cm.nblk - cb);
        const VT *pv = sv + k * (ST::VBYTES / (int)sizeof(VT));
        const IT *pc = sc + k * (ST::CBYTES / (int)sizeof(IT));
        const int xbase = sizeof(IT) == 2 ? cm.colbase : 0;  // base of the 16-bit offsets
        const VT *xb = x + xbase;
        const int xlo = -xbase, xhi = n - xbase;
        // blocks from pad_from on hold padding: their gathers test each column
        const int pad_from = (cm.flags & 1u) ? (int)(cm.flags >> 1) - cb : INT_MAX;
        auto gather4 = [&](const CBlk<IT> &cbk, VT (&xs)[4], int i) {
            if (i >= pad_from) {
#pragma unroll
                for (int q = 0; q < 4; ++q) xs[q] = cbk.gather(q, xb, pl, xlo, xhi, err);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) xs[q] = cbk.gather_all(q, xb, pl, xlo, xhi, err);
            }
        };
        VT xs[2][4];
        gather4(CBlk<IT>::load_smem(pc, 0, lane), xs[0], 0);
#pragma unroll
        for (int i = 0; i < KB; ++i) {
            if (i < len) {
                if (i + 1 < len)
                    gather4(CBlk<IT>::load_smem(pc, i + 1, lane), xs[(i + 1) & 1], i + 1);
                const VBlk<VT> vv = VBlk<VT>::load_smem(pv, i, lane);
#pragma unroll
                for (int q = 0; q < 4; ++q) acc.add(vv.get(q), xs[i & 1][q]);
            }
        }
        cb += KB;
        if (cb >= cm.nblk) {  // the slice's last piece
            const long long r = cs * 32 + lane;
            if (r < m) y[r] = acc.value();
            acc.reset();
            cb = 0;
            cs += nwarps;
            skip_empty();
        }
        __syncwarp();  // every lane is done with stage k
        if (ps < nslices) { issue(k); ++pending; }
        k = k + 1 == STAGES ? 0 : k + 1;
    }
    // only after a wait gave up: let the copies still in flight land before the CTA exits
    for (; pending > 0; --pending) {
        mbar_wait(bar0 + 8 * k, (phases >> k) & 1u);
        phases ^= 1u << k;
        k = k + 1 == STAGES ? 0 : k + 1;
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
    using ST = Stage<VT, IT>;
    // more than the default 48 KB of dynamic shared memory: opted into once per device
    static std::atomic<unsigned long long> opted{0};
    if (h.device < 0 || h.device >= 64) return cudaErrorInvalidDevice;
    const unsigned long long bit = 1ull << h.device;
    if (!(opted.load() & bit)) {
        const cudaError_t e = cudaFuncSetAttribute(
            sell_spmv_kernel<VT, IT>, cudaFuncAttributeMaxDynamicSharedMemorySize, ST::CTA_BYTES);
        if (e != cudaSuccess) return e;
        opted.fetch_or(bit);
    }
    const long long want = (h.nchunks + SELL_WARPS - 1) / SELL_WARPS;
    const long long cap = (long long)h.sm_count * CTAS_PER_SM;
    const unsigned grid = (unsigned)(want < cap ? want : cap);
    sell_spmv_kernel<VT, IT><<<grid, SELL_WARPS * 32, ST::CTA_BYTES, s>>>(
        (const SellSlice *)h.meta, (const VT *)h.vals, (const IT *)h.cols, (const VT *)x,
        (double *)y, h.nchunks, h.m, h.n, guard_word(), wait_word());
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
