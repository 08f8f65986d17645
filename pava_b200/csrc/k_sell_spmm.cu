// SELL SpMM: Y = A X for k right-hand sides (X row-major n x k, Y row-major m x k) on a SELL
// handle.
//
// A CTA of 32 G threads takes one 32-row slice at a time (slices in turn over the grid): G
// lanes per row (4, 8 or 16), 32 / G rows per warp.  Thread t owns row t / G of the slice and,
// of that row's k outputs, the KPL columns of slot g = t % G (VW = 2: the pairs g, g + G, ... of
// adjacent columns, each read as one vector) -- so the G lanes of a row read a whole row of X
// per nonzero, and each thread keeps its KPL sums in registers for the whole slice.
//
// The slice's value and column streams come into shared memory by bulk asynchronous copies
// (k_bulk.cuh), G blocks per piece, two pieces in flight per CTA: thread 0 issues the
// copies of the piece after next while the CTA sums the current one.  A row's four elements of
// a block are one 16-byte shared-memory read per stream (the G lanes of the row read the same
// address: a broadcast), where the row-group kernel (k_group.cu) passes every element to the
// lanes of its row by shuffles.  Padding elements (value 0, no column) read X row 0 and add
// nothing.
//
// No counterpart in the reference (its SpMV takes one vector; main.cpp:554-587 runs one matrix
// and one vector at a time).

#include <atomic>
#include <climits>
#include <cstdint>

#include "k_bulk.cuh"
#include "k_stream.cuh"
#include "pava_internal.h"

namespace pava {

namespace {

// The shape of G lanes per row: 32 G threads per CTA (32 rows), 32 / G CTAs per SM (32 warps),
// pieces of G blocks (about 100 KB of stages per SM for FP64 values and 32-bit columns, which
// leaves L1 room for the X rows neighbouring slices share; pieces of 2 G blocks were 5-10 %
// slower, of G / 2 blocks 4-7 % slower).
constexpr int SPMM_UNROLL = 2;  // blocks of a piece unrolled together
template <int G> struct SpmmShape {
    static_assert(G == 4 || G == 8 || G == 16, "lanes per row");
    static constexpr int THREADS = 32 * G, CTAS_PER_SM = 32 / G, KB = G;
};
template <typename VT, typename IT, int G> struct SpmmStage {
    static constexpr int VBYTES = SpmmShape<G>::KB * 128 * (int)sizeof(VT);
    static constexpr int CBYTES = SpmmShape<G>::KB * 128 * (int)sizeof(IT);
    static constexpr int BYTES = 2 * (VBYTES + CBYTES) + 128;  // two pieces + barriers
};

// Two adjacent columns of an X row in one read (16 bytes FP64, 8 bytes FP32), kept in L2.
__device__ __forceinline__ double2 ld_xpair(const double *p, uint64_t pol) {
    double2 r;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
                 : "=d"(r.x), "=d"(r.y) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ float2 ld_xpair(const float *p, uint64_t pol) {
    float2 r;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                 : "=f"(r.x), "=f"(r.y) : "l"(p), "l"(pol));
    return r;
}

// Column of sum p of a lane whose column slot is lg (0 .. G-1).
template <int G, int VW>
__device__ __forceinline__ int spmm_col(int lg, int p) {
    return VW == 1 ? lg + G * p : 2 * (lg + G * (p >> 1)) + (p & 1);
}

// The four elements of row r in block i of a shared-memory piece: columns (I32) or 16-bit
// offsets widened to int (DELTA_NONE stays -32768), and values.
__device__ __forceinline__ void row_cols(const int *pc, int i, int r, int (&c)[4]) {
    const int4 a = reinterpret_cast<const int4 *>(pc)[i * 32 + r];
    c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w;
}
__device__ __forceinline__ void row_cols(const short *pc, int i, int r, int (&c)[4]) {
    const uint2 a = reinterpret_cast<const uint2 *>(pc)[i * 32 + r];
    c[0] = (int)(a.x << 16) >> 16; c[1] = (int)a.x >> 16;
    c[2] = (int)(a.y << 16) >> 16; c[3] = (int)a.y >> 16;
}

template <typename VT, typename IT, int G, int KPL, int VW>
__global__ void __launch_bounds__(SpmmShape<G>::THREADS, SpmmShape<G>::CTAS_PER_SM)
sell_spmm_kernel(const SellSlice *__restrict__ meta, const VT *__restrict__ vals,
                 const IT *__restrict__ cols, const VT *__restrict__ X, long long ldx,
                 double *__restrict__ Y, long long ldy, long long nslices, int m, int n, int k,
                 unsigned long long *err, unsigned long long *wait_err) {
    using ST = SpmmStage<VT, IT, G>;
    constexpr int KB = SpmmShape<G>::KB;
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x;
    const int r = tid / G;   // the thread's row within the slice
    const int lg = tid % G;  // its column slot
    const unsigned bar0 = (unsigned)__cvta_generic_to_shared(smem);  // two barriers
    const VT *sv = reinterpret_cast<const VT *>(smem + 128);
    const IT *sc = reinterpret_cast<const IT *>(smem + 128 + 2 * ST::VBYTES);
    const unsigned sv0 = bar0 + 128, sc0 = bar0 + 128 + 2 * ST::VBYTES;
    if (tid == 0) {
        mbar_init(bar0);
        mbar_init(bar0 + 8);
        mbar_init_fence();
    }
    __syncthreads();
    const uint64_t pl = policy_evict_last();
    bool colok[KPL];
#pragma unroll
    for (int p = 0; p < KPL; ++p) colok[p] = spmm_col<G, VW>(lg, p) < k;
    // the CTA's slices, in turn over the grid (a contiguous run of slices per CTA, whose
    // neighbours share X rows, was measured slower on the stencil)
    const long long step = gridDim.x, s_first = blockIdx.x, s_end = nslices;

    // producer cursor (the CTA's slices with blocks; thread 0 issues the copies)
    long long ps = s_first;
    int pb = 0;
    SellSlice pm{0, 0, 0, 0u};
    auto p_find = [&]() {
        for (; ps < s_end; ps += step) {
            pm = meta[ps];
            if (pm.nblk > 0) break;
        }
    };
    p_find();
    auto issue = [&](int kk) {
        const int len = min(KB, pm.nblk - pb);
        const long long e0 = (long long)pm.off + (long long)pb * 128;
        if (tid == 0) {
            const unsigned vb = (unsigned)(len * 128 * (int)sizeof(VT));
            const unsigned cb = (unsigned)(len * 128 * (int)sizeof(IT));
            proxy_fence();  // the stage's last reads come before the copy's writes
            mbar_expect_tx(bar0 + 8 * kk, vb + cb);
            bulk_g2s(sv0 + kk * ST::VBYTES, vals + e0, vb, bar0 + 8 * kk);
            bulk_g2s(sc0 + kk * ST::CBYTES, cols + e0, cb, bar0 + 8 * kk);
        }
        pb += KB;
        if (pb >= pm.nblk) {
            pb = 0;
            ps += step;
            p_find();
        }
    };
    int pending = 0;
#pragma unroll
    for (int kk = 0; kk < 2; ++kk)
        if (ps < s_end) {
            issue(kk);
            ++pending;
        }

    // consumer cursor; the rows of empty slices are written as zeros
    long long cs = s_first;
    int cb = 0;
    SellSlice cm{0, 0, 0, 0u};
    auto store_row = [&](long long slice, const double (&acc)[KPL]) {
        const long long row = slice * 32 + r;
        if (row >= m) return;
        double *yr = Y + row * ldy;
#pragma unroll
        for (int p = 0; p < KPL; p += VW) {
            if (!colok[p]) continue;
            const int c = spmm_col<G, VW>(lg, p);
            if constexpr (VW == 2)
                *reinterpret_cast<double2 *>(yr + c) = make_double2(acc[p], acc[p + 1]);
            else
                yr[c] = acc[p];
        }
    };
    auto c_find = [&]() {
        double zero[KPL];
#pragma unroll
        for (int p = 0; p < KPL; ++p) zero[p] = 0.0;
        for (; cs < s_end; cs += step) {
            cm = meta[cs];
            if (cm.nblk > 0) break;
            store_row(cs, zero);
        }
    };
    c_find();
    unsigned phases = 0;  // bit kk: the parity awaited on stage kk
    int kk = 0;
    double acc[KPL];
#pragma unroll
    for (int p = 0; p < KPL; ++p) acc[p] = 0.0;
    while (cs < s_end) {
        // every thread waits (bounded); the CTA gives up together if any thread did
        const bool ok = mbar_wait(bar0 + 8 * kk, (phases >> kk) & 1u);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicAdd(&wait_err[0], 1ull);
                atomicCAS(&wait_err[1], 0ull, (unsigned long long)cs + 1);
            }
            break;
        }
        phases ^= 1u << kk;
        --pending;
        const int len = min(KB, cm.nblk - cb);
        const VT *pv = sv + kk * (ST::VBYTES / (int)sizeof(VT));
        const IT *pc = sc + kk * (ST::CBYTES / (int)sizeof(IT));
        const int xbase = sizeof(IT) == 2 ? cm.colbase : 0;  // base of the 16-bit offsets
#pragma unroll SPMM_UNROLL
        for (int i = 0; i < len; ++i) {
            int c[4];
            row_cols(pc, i, r, c);
            const VBlk<VT> vv = VBlk<VT>::load_smem(pv, i, r);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const bool real = sizeof(IT) == 2 ? c[q] != DELTA_NONE : c[q] >= 0;
                const int col = c[q] + xbase;
                const bool use = real && guard(err, col >= 0 && col < n, G_X, col);
                const VT *xr = X + (long long)(use ? col : 0) * ldx;  // row 0: a safe read
                const double v = (double)vv.get(q);
#pragma unroll
                for (int p = 0; p < KPL; p += VW) {
                    if (!colok[p]) continue;
                    const int cc = spmm_col<G, VW>(lg, p);
                    if constexpr (VW == 2) {
                        const auto x2 = ld_xpair(xr + cc, pl);
                        acc[p] = fma(v, use ? (double)x2.x : 0.0, acc[p]);
                        acc[p + 1] = fma(v, use ? (double)x2.y : 0.0, acc[p + 1]);
                    } else {
                        const VT xv = ld_x(xr + cc, pl);
                        acc[p] = fma(v, use ? (double)xv : 0.0, acc[p]);
                    }
                }
            }
        }
        cb += KB;
        if (cb >= cm.nblk) {  // the slice's last piece
            store_row(cs, acc);
#pragma unroll
            for (int p = 0; p < KPL; ++p) acc[p] = 0.0;
            cb = 0;
            cs += step;
            c_find();
        }
        __syncthreads();  // every thread is done with stage kk
        if (ps < s_end) {
            issue(kk);
            ++pending;
        }
        kk ^= 1;
    }
    // only after a wait gave up: let the copies still in flight land before the CTA exits
    for (; pending > 0; --pending) {
        mbar_wait(bar0 + 8 * kk, (phases >> kk) & 1u);
        phases ^= 1u << kk;
        kk ^= 1;
    }
}

template <typename VT, typename IT, int G, int KPL, int VW>
cudaError_t spmm_launch(const Handle &h, const VT *X, long long ldx, double *Y, long long ldy,
                        int k, cudaStream_t s) {
    using ST = SpmmStage<VT, IT, G>;
    // more than the default 48 KB of dynamic shared memory: opted into once per device
    static std::atomic<unsigned long long> opted{0};
    if (h.device < 0 || h.device >= 64) return cudaErrorInvalidDevice;
    const unsigned long long bit = 1ull << h.device;
    if (!(opted.load() & bit)) {
        const cudaError_t e = cudaFuncSetAttribute(sell_spmm_kernel<VT, IT, G, KPL, VW>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   ST::BYTES);
        if (e != cudaSuccess) return e;
        opted.fetch_or(bit);
    }
    const long long cap = (long long)h.sm_count * SpmmShape<G>::CTAS_PER_SM;
    const unsigned grid = (unsigned)(h.nchunks < cap ? h.nchunks : cap);
    sell_spmm_kernel<VT, IT, G, KPL, VW><<<grid, SpmmShape<G>::THREADS, ST::BYTES, s>>>(
        (const SellSlice *)h.meta, (const VT *)h.vals, (const IT *)h.cols, X, ldx, Y, ldy,
        h.nchunks, h.m, h.n, k, guard_word(), wait_word());
    return cudaGetLastError();
}

// KPL = the columns per lane that cover k with G lanes; pairs per read where they can be
template <typename VT, typename IT, int G, int KPL>
cudaError_t spmm_vw(const Handle &h, const VT *X, long long ldx, double *Y, long long ldy,
                    int k, cudaStream_t s) {
    const bool vec2 = KPL >= 2 && k % 2 == 0 && ldx % 2 == 0 && ldy % 2 == 0 &&
                      reinterpret_cast<uintptr_t>(X) % (2 * sizeof(VT)) == 0 &&
                      reinterpret_cast<uintptr_t>(Y) % 16 == 0;
    if constexpr (KPL >= 2)
        if (vec2) return spmm_launch<VT, IT, G, KPL, 2>(h, X, ldx, Y, ldy, k, s);
    return spmm_launch<VT, IT, G, KPL, 1>(h, X, ldx, Y, ldy, k, s);
}

template <typename VT, typename IT>
cudaError_t spmm_k(const Handle &h, const VT *X, long long ldx, double *Y, long long ldy, int k,
                   cudaStream_t s) {
    const int g = sell_spmm_lanes(h.lanes_per_row, k);
    if (g == 4) {
        if (k <= 4) return spmm_vw<VT, IT, 4, 1>(h, X, ldx, Y, ldy, k, s);
        if (k <= 8) return spmm_vw<VT, IT, 4, 2>(h, X, ldx, Y, ldy, k, s);
        if (k <= 16) return spmm_vw<VT, IT, 4, 4>(h, X, ldx, Y, ldy, k, s);
        if (k <= 32) return spmm_vw<VT, IT, 4, 8>(h, X, ldx, Y, ldy, k, s);
    } else if (g == 8) {
        if (k <= 8) return spmm_vw<VT, IT, 8, 1>(h, X, ldx, Y, ldy, k, s);
        if (k <= 16) return spmm_vw<VT, IT, 8, 2>(h, X, ldx, Y, ldy, k, s);
        if (k <= 32) return spmm_vw<VT, IT, 8, 4>(h, X, ldx, Y, ldy, k, s);
        if (k <= 64) return spmm_vw<VT, IT, 8, 8>(h, X, ldx, Y, ldy, k, s);
    } else if (g == 16) {
        if (k <= 16) return spmm_vw<VT, IT, 16, 1>(h, X, ldx, Y, ldy, k, s);
        if (k <= 32) return spmm_vw<VT, IT, 16, 2>(h, X, ldx, Y, ldy, k, s);
        if (k <= 64) return spmm_vw<VT, IT, 16, 4>(h, X, ldx, Y, ldy, k, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t sell_spmm(const Handle &h, const void *X, long long ldx, void *Y, long long ldy,
                      int k, cudaStream_t s) {
    if (h.nchunks <= 0 || k <= 0) return cudaSuccess;
    if (k > SELL_SPMM_MAX_K) return cudaErrorInvalidValue;
    const bool f32 = h.precision == PAVA_PREC_FP32C, d16 = h.index_mode == PAVA_INDEX_DELTA16;
    double *y = (double *)Y;
    if (!f32 && !d16) return spmm_k<double, int>(h, (const double *)X, ldx, y, ldy, k, s);
    if (!f32 && d16) return spmm_k<double, short>(h, (const double *)X, ldx, y, ldy, k, s);
    if (f32 && !d16) return spmm_k<float, int>(h, (const float *)X, ldx, y, ldy, k, s);
    return spmm_k<float, short>(h, (const float *)X, ldx, y, ldy, k, s);
}

}  // namespace pava
