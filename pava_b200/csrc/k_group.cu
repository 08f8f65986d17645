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

#include <climits>
#include <cstdint>
#include <type_traits>

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

// Rows shared by several column lanes (KCT = KC > 1, a compile-time count so that the KC
// elements of a round unroll): the group loads its row's nonzeros
// cooperatively, GL at a time (lane gi loads element base + gi, one coalesced load per lane and
// stream), with the next round's loads in flight while the current round is consumed; each
// element reaches the lanes that need it by shuffle.  Slice e takes elements e, e + ES, ... in
// ascending order, as the per-lane loop does, so the sums have the same bits.  The round count
// is the maximum over the warp's groups so that every shuffle has all 32 lanes.
template <int KPL, int KCT, int VW, typename VT, typename XREAD>
__device__ __forceinline__ void coop_row(int a, int b, int gi, int gl, int es, int e, int kc,
                                         int lane, const int *__restrict__ ci,
                                         const VT *__restrict__ v, const bool (&colok)[KPL],
                                         XREAD xread, Acc<VT> (&acc)[KPL], uint64_t pf) {
    int rounds = (b - a + gl - 1) / gl;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int t = __shfl_xor_sync(FULL, rounds, o);
        rounds = t > rounds ? t : rounds;
    }
    const int gbase = lane & ~(gl - 1);
    VT pv = VT(0);
    int pc = 0;
    if (a + gi < b) {
        pv = ld_val(v + a + gi, pf);
        pc = ld_col(ci + a + gi, pf);
    }
    for (int rd = 0; rd < rounds; ++rd) {
        const VT cv = pv;
        const int cc = pc;
        const int base = a + rd * gl;
        if (base + gl + gi < b) {  // next round in flight
            pv = ld_val(v + base + gl + gi, pf);
            pc = ld_col(ci + base + gl + gi, pf);
        }
#pragma unroll
        for (int u = 0; u < KCT; ++u) {
            const int o = e + u * es;
            const VT val = __shfl_sync(FULL, cv, gbase + o);
            const int col = __shfl_sync(FULL, cc, gbase + o);
            if (base + o < b) {
#pragma unroll
                for (int q = 0; q < KPL / VW; ++q)
                    if (colok[q * VW]) xread(col, q, val, acc);
            }
        }
    }
}

// Two adjacent right-hand sides of X in one 16-byte (8-byte for FP32) read.
__device__ __forceinline__ double2 ld_x2(const double *p, uint64_t pol) {
    double2 r;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
                 : "=d"(r.x), "=d"(r.y) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ float2 ld_x2(const float *p, uint64_t pol) {
    float2 r;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                 : "=f"(r.x), "=f"(r.y) : "l"(p), "l"(pol));
    return r;
}

// Column of accumulator p of a lane whose first column slot is cl: VW = 1 interleaves single
// columns across the KC lanes (cl + p KC); VW = 2 interleaves pairs (2 (cl + (p/2) KC) + p%2),
// so that a lane reads its two columns with one vector load and a group's KC lanes read
// 16 KC contiguous bytes.
template <int VW>
__device__ __forceinline__ int col_of(int cl, int p, int kc) {
    return VW == 1 ? cl + p * kc : 2 * (cl + (p >> 1) * kc) + (p & 1);
}

constexpr int GROUP_THREADS = 256;
// resident blocks per SM: more warps in flight for the narrow shapes
template <int KPL> constexpr int group_minb() { return KPL == 1 ? 6 : (KPL == 2 ? 5 : 4); }
// resident blocks per SM of the cooperative (k > 1) shapes
constexpr int COOP_MINB = 4;
// elements in flight per lane
template <int KPL> constexpr int group_unroll() { return KPL == 1 ? 4 : (KPL == 2 ? 2 : 1); }

template <int KPL, typename VT, int KCT, int VW>
__global__ void __launch_bounds__(GROUP_THREADS, KCT ? COOP_MINB : group_minb<KPL>())
csr_group_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                 const VT *__restrict__ v, const VT *__restrict__ X, long long ldx,
                 double *__restrict__ Y, long long ldy, int m, int k, int gl_shift,
                 int kc_shift, int tile_rows, int n, unsigned long long *err) {
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
    for (int p = 0; p < KPL; ++p) colok[p] = col_of<VW>(cl, p, kc) < k;
    // reads the VW columns of slot q of X row `col` and accumulates them
    auto xread = [&](int col, int q, VT val, Acc<VT>(&acc)[KPL]) {
        if (!guard(err, col >= 0 && col < n, G_X, col)) return;
        const VT *xr = X + (long long)col * ldx + col_of<VW>(cl, q * VW, kc);
        if (VW == 2) {
            const auto x2 = ld_x2(xr, pl);
            acc[2 * q].add(val, x2.x);
            acc[2 * q + 1].add(val, x2.y);
        } else {
            acc[q].add(val, ld_x(xr, pl));
        }
    };

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
            if (KCT) {
                coop_row<KPL, KCT, VW>(a, b, gi, gl, es, e, kc, lane, ci, v, colok, xread, acc,
                                       pf);
                j = b;
            }
            // U elements at a time (the last batch predicated): all value and column loads
            // first, then all gathers, so up to U memory round trips overlap even on short rows
            for (; j < b; j += U * es) {
                VT val[U];
                int col[U];
                bool in[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    in[u] = j + u * es < b;
                    val[u] = in[u] ? ld_val(v + j + u * es, pf) : VT(0);
                    col[u] = in[u] ? ld_col(ci + j + u * es, pf) : 0;
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < KPL / VW; ++q)
                        if (in[u] && colok[q * VW]) xread(col[u], q, val[u], acc);
            }
#pragma unroll
            for (int p = 0; p < KPL; ++p) {
                double s = acc[p].value();
                for (int o = kc; o < gl; o <<= 1) s += __shfl_xor_sync(FULL, s, o);
                if (valid && e == 0 && colok[p]) Y[r * ldy + col_of<VW>(cl, p, kc)] = s;
            }
        }
    }
}

// Windowed variant for k > 1 on matrices whose rows reach a narrow column range (banded,
// stencil-like): a CTA owns a tile of TR consecutive rows, finds the tile's column window
// [cmin, cmax], copies X[cmin .. cmax][0 .. k) into shared memory once, and its row groups
// read X from there.  Each X row is then fetched from L2 once per tile instead of once per
// nonzero that references it.  Tiles whose window does not fit take the global gathers.
constexpr int WINDOW_MINB = 2;
constexpr int WINDOW_SMEM = 100 * 1024;  // bytes of X per CTA (two CTAs per SM)

template <int KPL, typename VT, int KCT>
__global__ void __launch_bounds__(GROUP_THREADS, WINDOW_MINB)
csr_window_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                  const VT *__restrict__ v, const VT *__restrict__ X, long long ldx,
                  double *__restrict__ Y, long long ldy, int m, int k, int gl_shift,
                  int kc_shift, int tile_rows, int max_w, int n, unsigned long long *err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    VT *xs = reinterpret_cast<VT *>(smem_raw);
    constexpr int WARPS = GROUP_THREADS / 32;
    __shared__ int s_min[WARPS], s_max[WARPS];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int gl = 1 << gl_shift, kc = 1 << kc_shift;
    const int grp = lane >> gl_shift;
    const int gpw = 32 >> gl_shift;
    const int gi = lane & (gl - 1);
    const int e = gi >> kc_shift;
    const int es = gl >> kc_shift;
    const int cl = gi & (kc - 1);
    const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
    const long long ntiles = ((long long)m + tile_rows - 1) / tile_rows;
    const int rows_per_pass = WARPS * gpw;

    bool colok[KPL];
#pragma unroll
    for (int p = 0; p < KPL; ++p) colok[p] = cl + p * kc < k;

    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long r0 = t * tile_rows;
        const long long r1 = r0 + tile_rows < m ? r0 + tile_rows : m;
        // the tile's column window
        const int j0 = rp[r0], j1 = rp[r1];
        int cmin = INT_MAX, cmax = -1;
        for (int j = j0 + tid; j < j1; j += GROUP_THREADS) {
            const int c = ci[j];
            cmin = c < cmin ? c : cmin;
            cmax = c > cmax ? c : cmax;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int a = __shfl_xor_sync(FULL, cmin, o), b = __shfl_xor_sync(FULL, cmax, o);
            cmin = a < cmin ? a : cmin;
            cmax = b > cmax ? b : cmax;
        }
        if (lane == 0) {
            s_min[w] = cmin;
            s_max[w] = cmax;
        }
        __syncthreads();
        cmin = s_min[0];
        cmax = s_max[0];
#pragma unroll
        for (int q = 1; q < WARPS; ++q) {
            cmin = s_min[q] < cmin ? s_min[q] : cmin;
            cmax = s_max[q] > cmax ? s_max[q] : cmax;
        }
        const int W = cmax >= cmin ? cmax - cmin + 1 : 0;
        const bool staged = W > 0 && W <= max_w &&
                            guard(err, cmin >= 0 && cmax < n, G_X, cmin < 0 ? cmin : cmax);
        if (staged) {  // X[cmin .. cmax][0 .. k) -> xs, row stride k; SU loads in flight
            constexpr int SU = 8;
            const int total = W * k;  // <= WINDOW_SMEM / sizeof(VT)
            const VT *src = X + (long long)cmin * ldx;
            for (int q0 = tid; q0 < total; q0 += SU * GROUP_THREADS) {
                VT t[SU];
#pragma unroll
                for (int u = 0; u < SU; ++u) {
                    const int q = q0 + u * GROUP_THREADS;
                    if (q < total) {
                        if (ldx == k) {
                            t[u] = ld_x(src + q, pl);
                        } else {
                            const int wr = q / k;
                            t[u] = ld_x(src + (long long)wr * ldx + (q - wr * k), pl);
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < SU; ++u) {
                    const int q = q0 + u * GROUP_THREADS;
                    if (q < total) xs[q] = t[u];
                }
            }
        }
        __syncthreads();
        for (long long rb = r0; rb < r1; rb += rows_per_pass) {
            const long long r = rb + (long long)w * gpw + grp;
            const bool valid = r < r1;
            int a = 0, b = 0;
            if (valid) {
                a = rp[r];
                b = rp[r + 1];
            }
            Acc<VT> acc[KPL];
            int j = a + e;
            if (KCT) {
                if (staged)
                    coop_row<KPL, KCT, 1>(
                        a, b, gi, gl, es, e, kc, lane, ci, v, colok,
                        [&](int col, int p, VT val, Acc<VT>(&ac)[KPL]) {
                            ac[p].add(val, xs[(col - cmin) * k + cl + p * kc]);
                        },
                        acc, pf);
                else
                    coop_row<KPL, KCT, 1>(
                        a, b, gi, gl, es, e, kc, lane, ci, v, colok,
                        [&](int col, int p, VT val, Acc<VT>(&ac)[KPL]) {
                            if (guard(err, col >= 0 && col < n, G_X, col))
                                ac[p].add(val, ld_x(X + (long long)col * ldx + cl + p * kc, pl));
                        },
                        acc, pf);
                j = b;
            } else if (staged) {  // WU elements' values and columns in flight, then the shared reads
                constexpr int WU = 4;
                for (; j + (WU - 1) * es < b; j += WU * es) {
                    VT val[WU];
                    int col[WU];
#pragma unroll
                    for (int u = 0; u < WU; ++u) {
                        val[u] = ld_val(v + j + u * es, pf);
                        col[u] = ld_col(ci + j + u * es, pf);
                    }
#pragma unroll
                    for (int u = 0; u < WU; ++u) {
                        const VT *xr = xs + (col[u] - cmin) * k + cl;
#pragma unroll
                        for (int p = 0; p < KPL; ++p)
                            if (colok[p]) acc[p].add(val[u], xr[p * kc]);
                    }
                }
            }
            for (; j < b; j += es) {
                const VT val = ld_val(v + j, pf);
                const int col = ld_col(ci + j, pf);
                if (staged) {
                    const VT *xr = xs + (col - cmin) * k + cl;
#pragma unroll
                    for (int p = 0; p < KPL; ++p)
                        if (colok[p]) acc[p].add(val, xr[p * kc]);
                } else if (guard(err, col >= 0 && col < n, G_X, col)) {
                    const VT *xr = X + (long long)col * ldx + cl;
#pragma unroll
                    for (int p = 0; p < KPL; ++p)
                        if (colok[p]) acc[p].add(val, ld_x(xr + p * kc, pl));
                }
            }
#pragma unroll
            for (int p = 0; p < KPL; ++p) {
                double s = acc[p].value();
                for (int o = kc; o < gl; o <<= 1) s += __shfl_xor_sync(FULL, s, o);
                if (valid && e == 0 && colok[p]) Y[r * ldy + cl + p * kc] = s;
            }
        }
        __syncthreads();  // xs is restaged by the next tile
    }
}

int ilog2(int v) {
    int s = 0;
    while ((1 << s) < v) ++s;
    return s;
}

// Calls f(std::integral_constant<int, KC>) for the column-lane count kc (1 = not cooperative).
template <typename F>
cudaError_t with_kc(int kc, F f) {
    switch (kc) {
        case 1: return f(std::integral_constant<int, 0>());
        case 2: return f(std::integral_constant<int, 2>());
        case 4: return f(std::integral_constant<int, 4>());
        case 8: return f(std::integral_constant<int, 8>());
        case 16: return f(std::integral_constant<int, 16>());
        case 32: return f(std::integral_constant<int, 32>());
        default: return cudaErrorInvalidValue;
    }
}

template <int KPL, typename VT>
cudaError_t launch_window(const Handle &h, const VT *x, long long ldx, double *y, long long ldy,
                          int k, cudaStream_t s) {
    const int tr = h.rows_per_tile;
    const long long ntiles = ((long long)h.m + tr - 1) / tr;
    const long long cap = (long long)h.sm_count * WINDOW_MINB;
    const unsigned grid = (unsigned)(ntiles < cap ? (ntiles > 0 ? ntiles : 1) : cap);
    const int max_w = (int)(WINDOW_SMEM / ((size_t)k * sizeof(VT)));
    const size_t smem = (size_t)max_w * k * sizeof(VT);
    return with_kc(h.col_lanes, [&](auto KCC) {
        constexpr int KCT = decltype(KCC)::value;
        // per launch: the attribute belongs to the current device
        const cudaError_t attr = cudaFuncSetAttribute(
            csr_window_kernel<KPL, VT, KCT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
            WINDOW_SMEM);
        if (attr != cudaSuccess) return attr;
        csr_window_kernel<KPL, VT, KCT><<<grid, GROUP_THREADS, smem, s>>>(
            h.rp, h.ci, (const VT *)h.v, x, ldx, y, ldy, h.m, k, ilog2(h.lanes_per_row),
            ilog2(h.col_lanes), tr, max_w, h.n, guard_word());
        return cudaGetLastError();
    });
}

template <int KPL, typename VT>
cudaError_t launch_rows(const Handle &h, const VT *x, long long ldx, double *y, long long ldy,
                        int k, cudaStream_t s) {
    const int kc = h.col_lanes;
    const int tr = h.rows_per_tile;
    const long long ntiles = ((long long)h.m + tr - 1) / tr;
    const long long want = (ntiles + (GROUP_THREADS / 32) - 1) / (GROUP_THREADS / 32);
    const int minb = kc > 1 ? COOP_MINB : group_minb<KPL>();
    const long long cap = (long long)h.sm_count * minb;
    const unsigned grid = (unsigned)(want < cap ? (want > 0 ? want : 1) : cap);
    const int gs = ilog2(h.lanes_per_row), ks = ilog2(kc);
    // pairs of columns per vector read when every pair is whole and 2-element aligned
    const bool vec2 = KPL >= 2 && k % 2 == 0 && ldx % 2 == 0 &&
                      reinterpret_cast<uintptr_t>(x) % (2 * sizeof(VT)) == 0;
    return with_kc(kc, [&](auto KCC) {
        constexpr int KCT = decltype(KCC)::value;
        constexpr int VW2 = KPL >= 2 ? 2 : 1;
        if (vec2)
            csr_group_kernel<KPL, VT, KCT, VW2><<<grid, GROUP_THREADS, 0, s>>>(
                h.rp, h.ci, (const VT *)h.v, x, ldx, y, ldy, h.m, k, gs, ks, tr, h.n,
                guard_word());
        else
            csr_group_kernel<KPL, VT, KCT, 1><<<grid, GROUP_THREADS, 0, s>>>(
                h.rp, h.ci, (const VT *)h.v, x, ldx, y, ldy, h.m, k, gs, ks, tr, h.n,
                guard_word());
        return cudaGetLastError();
    });
}

template <typename VT>
cudaError_t launch_group(const Handle &h, const void *X, long long ldx, void *Y, long long ldy,
                         int k, cudaStream_t s) {
    const VT *x = (const VT *)X;
    double *y = (double *)Y;
    if (h.x_window) {
        switch (h.cols_per_lane) {
            case 1: return launch_window<1, VT>(h, x, ldx, y, ldy, k, s);
            case 2: return launch_window<2, VT>(h, x, ldx, y, ldy, k, s);
            case 4: return launch_window<4, VT>(h, x, ldx, y, ldy, k, s);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (h.cols_per_lane) {
        case 1: return launch_rows<1, VT>(h, x, ldx, y, ldy, k, s);
        case 2: return launch_rows<2, VT>(h, x, ldx, y, ldy, k, s);
        case 4: return launch_rows<4, VT>(h, x, ldx, y, ldy, k, s);
        default: return cudaErrorInvalidValue;
    }
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
