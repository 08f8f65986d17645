// Shared device helpers for the pava B200 SpMV engine (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pava {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned r;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
    return r;
}

// L2 policies: the format streams (values, columns, flags) are read once per SpMV and are
// marked evict-first so that x, which every SpMV gathers from, stays resident in L2.
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ double2 ld_stream(const double2 *p, uint64_t pol) {
    double2 r;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;"
                 : "=d"(r.x), "=d"(r.y) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ float4 ld_stream(const float4 *p, uint64_t pol) {
    float4 r;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ int4 ld_stream(const int4 *p, uint64_t pol) {
    int4 r;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ uint2 ld_stream(const uint2 *p, uint64_t pol) {
    uint2 r;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0,%1}, [%2], %3;"
                 : "=r"(r.x), "=r"(r.y) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ unsigned ld_stream(const unsigned *p, uint64_t pol) {
    unsigned r;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;"
                 : "=r"(r) : "l"(p), "l"(pol));
    return r;
}

// x gather: read-only path through L1 (stencil rows reuse neighbours' x), kept in L2.
__device__ __forceinline__ double ld_x(const double *p, uint64_t pol) {
    double r;
    asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(r) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ float ld_x(const float *p, uint64_t pol) {
    float r;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(r) : "l"(p), "l"(pol));
    return r;
}

// Last index r in [0, n) with a[r] <= key (a sorted ascending, a[0] <= key).
__device__ __forceinline__ int upper_bound_m1(const int *a, int n, long long key) {
    int lo = 0, hi = n;  // first index with a[idx] > key lies in [lo, hi]
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if ((long long)a[mid] <= key) lo = mid + 1; else hi = mid;
    }
    return lo - 1;
}

// Fixed-order warp sum (xor butterfly): every lane gets the same bits on every run.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(FULL, v, d);
    return v;
}

// Segmented suffix combine over lanes: H_k = a_k + (pass_k ? H_{k+1} : 0), H_32 = 0.
// Kogge-Stone on the pairs (a, pass); the tree is fixed, so results are bitwise repeatable.
__device__ __forceinline__ double seg_suffix(double a, bool pass, int lane) {
    unsigned p = pass ? 1u : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        double an = __shfl_down_sync(FULL, a, d);
        unsigned pn = __shfl_down_sync(FULL, p, d);
        if (lane + d < 32) {
            if (p) a += an;
            p &= pn;
        }
    }
    return a;
}

__device__ __forceinline__ int warp_excl_scan(int v, int lane) {
    int s = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int t = __shfl_up_sync(FULL, s, d);
        if (lane >= d) s += t;
    }
    return s - v;
}

// ---- bounds-checked builds ---------------------------------------------------------------
// Built with -DPAVA_BOUNDS_CHECK (python -m pava_b200.build --bounds), the SpMV kernels test
// every index that comes from data before they use it -- the column of each x gather, the row
// of each y store, slot numbers read from the format's metadata, the carry chunk of a shared
// row.  A failed test increments the error word err[0] (the first failure also leaves its site
// in err[1] and the index in err[2]) and the access is skipped, so a bad index becomes a
// status the host reads (pava_bounds_report) instead of a fault.  In ordinary builds the tests
// compile to nothing.
enum GuardSite : unsigned {
    G_X = 1,      // x gather column outside [0, n)
    G_Y = 2,      // y row outside [0, m)
    G_CARRY = 3,  // carry chunk outside [0, nchunks)
    G_SLOT = 4,   // shared-memory slot or tail count from the metadata outside its array
};

__device__ __forceinline__ bool guard(unsigned long long *err, bool ok, unsigned site,
                                      long long idx) {
#ifdef PAVA_BOUNDS_CHECK
    if (!ok && err) {
        if (atomicAdd(err, 1ull) == 0ull) {
            err[1] = site;
            err[2] = (unsigned long long)idx;
        }
    }
    return ok;
#else
    (void)err; (void)ok; (void)site; (void)idx;
    return true;
#endif
}

// Common prefix of every chunk's metadata: rows the chunk touches and whether its first /
// last row continues into the neighbouring chunk.  The carry fixup reads only this prefix.
struct ChunkHdr {
    int r_first;      // row of the chunk's first element
    int nrows;        // r_last - r_first + 1
    unsigned shared;  // bit0: r_first began in an earlier chunk; bit1: r_last continues after
    int aux;
};

// Writes a finished row sum: the chunk's shared first / last rows go to the carry slots that
// the fixup pass combines in chunk order; every other row is stored straight into y.  Rows
// >= m belong to the virtual row that pads the last chunk and are dropped.
template <typename YT>
__device__ __forceinline__ void flush_row(int row, double val, int r_first, int r_last,
                                          unsigned shared, long long c, YT *y,
                                          double *carry_head, double *carry_tail, int m,
                                          unsigned long long *err = nullptr) {
    if (row == r_first && (shared & 1u)) carry_head[c] = val;
    else if (row == r_last && (shared & 2u)) carry_tail[c] = val;
    else if (row < m && guard(err, row >= 0, G_Y, row)) y[row] = (YT)val;
}

}  // namespace pava
