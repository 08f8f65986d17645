// Stream blocks shared by the CVR and CSR5 SpMV kernels.
//
// Both formats store a warp chunk as a sequence of 4-step blocks of 128 elements: element
// (step i, lane k) of block b sits at chunk_base + b*128 + 4k + (i%4) for values held as FP32
// or columns of either width, and at chunk_base + b*128 + 64*(i%4 / 2) + 2k + (i%2) for FP64
// values.  Each lane therefore reads one 16-byte vector per block per stream (8 bytes for the
// 16-bit columns), and a warp reads whole 128-byte lines.
//
// Value forms:  double -- FP64 values and x, FMA accumulation;
//               float  -- FP32 values and x, compensated accumulation (TwoProduct by FMA,
//                         TwoSum), the sum and its correction widened to FP64 at the end.
// Column forms: int    -- 32-bit columns;
//               short  -- 16-bit offsets from the chunk's base column (col = base + d), with
//                         d = -32768 marking an element that reads no x.
#pragma once
#include "pava_common.cuh"

namespace pava {

constexpr short DELTA_NONE = -32768;

template <typename VT> struct VBlk;
template <> struct VBlk<double> {
    double2 a, b;
    __device__ __forceinline__ double get(int q) const {
        return q == 0 ? a.x : q == 1 ? a.y : q == 2 ? b.x : b.y;
    }
    __device__ __forceinline__ static VBlk load(const double *base, int blk, int lane, uint64_t pol) {
        const double2 *p = reinterpret_cast<const double2 *>(base);
        VBlk r;
        r.a = ld_stream(p + (2 * blk) * 32 + lane, pol);
        r.b = ld_stream(p + (2 * blk + 1) * 32 + lane, pol);
        return r;
    }
    // the same block from a copy of the stream in shared memory
    __device__ __forceinline__ static VBlk load_smem(const double *base, int blk, int lane) {
        const double2 *p = reinterpret_cast<const double2 *>(base);
        VBlk r;
        r.a = p[(2 * blk) * 32 + lane];
        r.b = p[(2 * blk + 1) * 32 + lane];
        return r;
    }
};
template <> struct VBlk<float> {
    float4 a;
    __device__ __forceinline__ float get(int q) const {
        return q == 0 ? a.x : q == 1 ? a.y : q == 2 ? a.z : a.w;
    }
    __device__ __forceinline__ static VBlk load(const float *base, int blk, int lane, uint64_t pol) {
        VBlk r;
        r.a = ld_stream(reinterpret_cast<const float4 *>(base) + blk * 32 + lane, pol);
        return r;
    }
    __device__ __forceinline__ static VBlk load_smem(const float *base, int blk, int lane) {
        VBlk r;
        r.a = reinterpret_cast<const float4 *>(base)[blk * 32 + lane];
        return r;
    }
};

template <typename IT> struct CBlk;
template <> struct CBlk<int> {
    // x of element q: xb is x itself for 32-bit columns.  Column -1 (the dummy element of an
    // empty row, or chunk padding) reads nothing and gives 0, so a non-finite x never leaks
    // into an empty row.
    // [xlo, xhi): the indices of xb that lie in x (tested in bounds-checked builds only)
    template <typename T>
    __device__ __forceinline__ T gather(int q, const T *xb, uint64_t pol, int xlo = 0,
                                        int xhi = 0, unsigned long long *err = nullptr) const {
        const int c = col(q, 0);
        if (c < 0 || !guard(err, c >= xlo && c < xhi, G_X, c)) return T(0);
        return ld_x(xb + c, pol);
    }
    // the same where every element of the chunk reads x
    template <typename T>
    __device__ __forceinline__ T gather_all(int q, const T *xb, uint64_t pol, int xlo = 0,
                                            int xhi = 0, unsigned long long *err = nullptr) const {
        const int c = col(q, 0);
        if (!guard(err, c >= xlo && c < xhi, G_X, c)) return T(0);
        return ld_x(xb + c, pol);
    }
    int4 a;
    __device__ __forceinline__ int col(int q, int) const {
        return q == 0 ? a.x : q == 1 ? a.y : q == 2 ? a.z : a.w;
    }
    __device__ __forceinline__ static CBlk load(const int *base, int blk, int lane, uint64_t pol) {
        CBlk r;
        r.a = ld_stream(reinterpret_cast<const int4 *>(base) + blk * 32 + lane, pol);
        return r;
    }
    __device__ __forceinline__ static CBlk load_smem(const int *base, int blk, int lane) {
        CBlk r;
        r.a = reinterpret_cast<const int4 *>(base)[blk * 32 + lane];
        return r;
    }
};
template <> struct CBlk<short> {
    // x of element q: xb = x + (the chunk's base column); the offset DELTA_NONE reads nothing
    template <typename T>
    __device__ __forceinline__ T gather(int q, const T *xb, uint64_t pol, int xlo = 0,
                                        int xhi = 0, unsigned long long *err = nullptr) const {
        const unsigned w = q < 2 ? a.x : a.y;
        const int d = (q & 1) ? ((int)w >> 16) : ((int)(w << 16) >> 16);
        if (d == DELTA_NONE || !guard(err, d >= xlo && d < xhi, G_X, d)) return T(0);
        return ld_x(xb + d, pol);
    }
    template <typename T>
    __device__ __forceinline__ T gather_all(int q, const T *xb, uint64_t pol, int xlo = 0,
                                            int xhi = 0, unsigned long long *err = nullptr) const {
        const unsigned w = q < 2 ? a.x : a.y;
        const int d = (q & 1) ? ((int)w >> 16) : ((int)(w << 16) >> 16);
        if (!guard(err, d >= xlo && d < xhi, G_X, d)) return T(0);
        return ld_x(xb + d, pol);
    }
    uint2 a;
    __device__ __forceinline__ int col(int q, int base) const {
        const unsigned w = q < 2 ? a.x : a.y;
        const int d = (q & 1) ? ((int)w >> 16) : ((int)(w << 16) >> 16);
        return d == DELTA_NONE ? -1 : base + d;
    }
    __device__ __forceinline__ static CBlk load(const short *base, int blk, int lane, uint64_t pol) {
        CBlk r;
        r.a = ld_stream(reinterpret_cast<const uint2 *>(base) + blk * 32 + lane, pol);
        return r;
    }
    __device__ __forceinline__ static CBlk load_smem(const short *base, int blk, int lane) {
        CBlk r;
        r.a = reinterpret_cast<const uint2 *>(base)[blk * 32 + lane];
        return r;
    }
};

// Element offset inside a chunk's value / column stream for (step i, lane k).
template <typename VT>
__host__ __device__ __forceinline__ long long vals_offset(int i, int k) {
    if (sizeof(VT) == 8) return (long long)(i >> 1) * 64 + 2 * k + (i & 1);
    return (long long)(i >> 2) * 128 + 4 * k + (i & 3);
}
__host__ __device__ __forceinline__ long long cols_offset(int i, int k) {
    return (long long)(i >> 2) * 128 + 4 * k + (i & 3);
}

template <typename VT> struct Acc;
// Predicated shared-memory stores and loads of a parked row piece (shared-window addresses).
__device__ __forceinline__ void sts_pred(unsigned addr, double v, bool p) {
    asm volatile("{ .reg .pred q; setp.ne.u32 q, %2, 0; @q st.shared.f64 [%0], %1; }"
                 :: "r"(addr), "d"(v), "r"((unsigned)p) : "memory");
}
__device__ __forceinline__ void sts_pred(unsigned addr, float a, float b, bool p) {
    asm volatile("{ .reg .pred q; setp.ne.u32 q, %3, 0; @q st.shared.v2.f32 [%0], {%1, %2}; }"
                 :: "r"(addr), "f"(a), "f"(b), "r"((unsigned)p) : "memory");
}
__device__ __forceinline__ double lds_f64(unsigned addr) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ float2 lds_v2f32(unsigned addr) {
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
    return v;
}

// Row accumulators.  push parks the current piece at a shared address when p is set,
// piece_at reads one back as FP64, add_restart(v, x, st) starts a new sum at v*x when st is set.
template <> struct Acc<double> {
    __device__ __forceinline__ void push(unsigned addr, bool p) const { sts_pred(addr, s, p); }
    __device__ __forceinline__ static double piece_at(unsigned addr) { return lds_f64(addr); }
    __device__ __forceinline__ void add_restart(double v, double x, bool st) {
        s = fma(v, x, st ? 0.0 : s);
    }
    double s = 0.0;
    __device__ __forceinline__ void add(double v, double x) { s = fma(v, x, s); }
    __device__ __forceinline__ double value() const { return s; }
    __device__ __forceinline__ void reset() { s = 0.0; }
};
template <> struct Acc<float> {
    __device__ __forceinline__ void push(unsigned addr, bool p) const { sts_pred(addr, s, c, p); }
    __device__ __forceinline__ static double piece_at(unsigned addr) {
        const float2 v = lds_v2f32(addr);
        return (double)v.x + (double)v.y;
    }
    float s = 0.f, c = 0.f;
    // Every step rounds on its own (the _rn intrinsics are never contracted into an FMA),
    // which the exactness of TwoProduct and TwoSum relies on.
    __device__ __forceinline__ void add(float v, float x) {
        const float p = __fmul_rn(v, x);
        const float e = __fmaf_rn(v, x, -p);  // v*x = p + e exactly
        const float t = __fadd_rn(s, p);      // TwoSum(s, p) = t + err exactly
        const float z = __fsub_rn(t, s);
        const float err = __fadd_rn(__fsub_rn(s, __fsub_rn(t, z)), __fsub_rn(p, z));
        s = t;
        c = __fadd_rn(c, __fadd_rn(err, e));
    }
    __device__ __forceinline__ void add_restart(float v, float x, bool st) {
        s = st ? 0.f : s;
        c = st ? 0.f : c;
        add(v, x);
    }
    __device__ __forceinline__ double value() const { return (double)s + (double)c; }
    __device__ __forceinline__ void reset() { s = 0.f; c = 0.f; }
};

__device__ __forceinline__ unsigned ld_flag(const unsigned *p) {
    unsigned r;
    asm volatile("ld.global.nc.u32 %0, [%1];" : "=r"(r) : "l"(p));
    return r;
}

}  // namespace pava
