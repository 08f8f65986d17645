// Floor kernels: the two costs an SpMV on a matrix with scattered columns is made of, measured
// apart, so that an SpMV kernel's time can be held against max(stream floor, gather floor).
//
// Each kernel walks nnz elements in CSR order, four consecutive elements per thread per step
// (16-byte loads of the column stream, two of the value stream, with the same L2 policies as
// the SpMV kernels: streams evict-first and not kept in L1, x evict-last), and reduces what it
// read into one double per warp so that no load can be dropped.  No rows, no flags, no
// carries: what the SpMV adds on top of these is the cost of its row structure.
//
//   STREAMS  values and columns read, no x:            sum v * (double)c   12 B per element
//   GATHERS  x at columns drawn by a hash, no streams:  sum x[h(i) mod n]   one 8-byte gather
//   COLGATH  the column stream and x at those columns:  sum x[c]            4 B + one gather
//   DOT      values, columns and x at the columns:      sum v * x[c]        12 B + one gather
//   TMAGATH  GATHERS' x values fetched by the TMA engine instead of the load units: x viewed as
//            n / 2 rows of 16 bytes under a 2-D tensor map, lanes 0..7 of a warp each issue one
//            cp.async.bulk.tensor tile::gather4 (four rows, box one row high) per 32 elements
//            into shared memory, completion on an mbarrier (bounded waits), lane l then reads
//            its value there -- the other gather path of sm_100, measured beside the L1 one
//
// No counterpart in the reference: a measurement aid only (pava_probe.h).

#include <cuda.h>
#include <cudaTypedefs.h>

#include "../../include/pava_probe.h"
#include "k_bulk.cuh"
#include "pava_common.cuh"

namespace pava {
namespace {

enum { STREAMS = 0, GATHERS = 1, COLGATH = 2, DOT = 3, TMAGATH = 4 };

__device__ __forceinline__ unsigned hash_col(unsigned long long i, unsigned long long seed,
                                             unsigned n) {
    unsigned long long z = i + seed * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (unsigned)(((z >> 32) * (unsigned long long)n) >> 32);
}

template <int MODE>
__global__ void floor_kernel(const double *__restrict__ vals, const int *__restrict__ cols,
                             const double *__restrict__ x, long long nnz, int n,
                             unsigned long long seed, double *__restrict__ out) {
    const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long ngroups = nnz >> 2;  // groups of four elements
    double acc = 0.0;
    // two groups per thread per iteration: 8 gathers and 3-6 stream vectors in flight
    long long g = tid;
    for (; g + nthreads < ngroups; g += 2 * nthreads) {
        const long long h = g + nthreads;
        int4 c0 = make_int4(0, 0, 0, 0), c1 = make_int4(0, 0, 0, 0);
        double2 a0 = make_double2(0, 0), b0 = a0, a1 = a0, b1 = a0;
        if (MODE != GATHERS) {
            c0 = ld_stream(reinterpret_cast<const int4 *>(cols) + g, pf);
            c1 = ld_stream(reinterpret_cast<const int4 *>(cols) + h, pf);
        }
        if (MODE == STREAMS || MODE == DOT) {
            a0 = ld_stream(reinterpret_cast<const double2 *>(vals) + 2 * g, pf);
            b0 = ld_stream(reinterpret_cast<const double2 *>(vals) + 2 * g + 1, pf);
            a1 = ld_stream(reinterpret_cast<const double2 *>(vals) + 2 * h, pf);
            b1 = ld_stream(reinterpret_cast<const double2 *>(vals) + 2 * h + 1, pf);
        }
        if (MODE == GATHERS) {
            c0 = make_int4(hash_col(4 * g, seed, n), hash_col(4 * g + 1, seed, n),
                           hash_col(4 * g + 2, seed, n), hash_col(4 * g + 3, seed, n));
            c1 = make_int4(hash_col(4 * h, seed, n), hash_col(4 * h + 1, seed, n),
                           hash_col(4 * h + 2, seed, n), hash_col(4 * h + 3, seed, n));
        }
        if (MODE == STREAMS) {
            acc += a0.x * c0.x + a0.y * c0.y + b0.x * c0.z + b0.y * c0.w;
            acc += a1.x * c1.x + a1.y * c1.y + b1.x * c1.z + b1.y * c1.w;
        } else {
            const double x0 = ld_x(x + c0.x, pl), x1 = ld_x(x + c0.y, pl);
            const double x2 = ld_x(x + c0.z, pl), x3 = ld_x(x + c0.w, pl);
            const double x4 = ld_x(x + c1.x, pl), x5 = ld_x(x + c1.y, pl);
            const double x6 = ld_x(x + c1.z, pl), x7 = ld_x(x + c1.w, pl);
            if (MODE == DOT) {
                acc = fma(a0.x, x0, acc); acc = fma(a0.y, x1, acc);
                acc = fma(b0.x, x2, acc); acc = fma(b0.y, x3, acc);
                acc = fma(a1.x, x4, acc); acc = fma(a1.y, x5, acc);
                acc = fma(b1.x, x6, acc); acc = fma(b1.y, x7, acc);
            } else {
                acc += ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
            }
        }
    }
    for (; g < ngroups; g += nthreads) {  // a last odd group
        for (int q = 0; q < 4; ++q) {
            const long long i = 4 * g + q;
            const int c = MODE == GATHERS ? (int)hash_col(i, seed, n) : cols[i];
            const double v = (MODE == STREAMS || MODE == DOT) ? vals[i] : 1.0;
            acc += MODE == STREAMS ? v * c : v * x[c];
        }
    }
    for (long long i = 4 * ngroups + tid; i < nnz; i += nthreads) {  // nnz % 4 tail
        const int c = MODE == GATHERS ? (int)hash_col(i, seed, n) : cols[i];
        const double v = (MODE == STREAMS || MODE == DOT) ? vals[i] : 1.0;
        acc += MODE == STREAMS ? v * c : v * x[c];
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) out[tid >> 5] = acc;
}

// TMAGATH: 8 warps per CTA; per warp and step 32 elements, eight gather4 pieces of 64 bytes
// (each at a 128-byte boundary) in one of two 1 KB slots, one mbarrier per slot.
constexpr int TMA_WARPS = 8;
__global__ void __launch_bounds__(TMA_WARPS * 32)
tma_gather_kernel(const __grid_constant__ CUtensorMap tmap, long long nnz, int n,
                  unsigned long long seed, double *__restrict__ out,
                  unsigned long long *__restrict__ wait_fail) {
    __shared__ __align__(128) unsigned char slots[TMA_WARPS][2][1024];
    __shared__ __align__(8) unsigned long long bars[TMA_WARPS][2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned bar0 = (unsigned)__cvta_generic_to_shared(&bars[w][0]);
    if (lane == 0) {
        mbar_init(bar0);
        mbar_init(bar0 + 8);
        mbar_init_fence();
    }
    __syncwarp();
    const long long nwarps = (long long)gridDim.x * TMA_WARPS;
    const long long wid = (long long)blockIdx.x * TMA_WARPS + w;
    const long long steps = nnz / 32;  // whole steps of 32 elements
    auto issue = [&](long long step, int b) {
        if (lane < 8) {
            const unsigned long long i0 = (unsigned long long)step * 32 + lane * 4;
            int rows[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) rows[j] = (int)(hash_col(i0 + j, seed, n) >> 1);
            const unsigned bar = bar0 + 8 * b;
            if (lane == 0) mbar_expect_tx(bar, 8 * 64);
            __syncwarp(0xffu);
            const unsigned dst = (unsigned)__cvta_generic_to_shared(&slots[w][b][lane * 128]);
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::"
                "complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
                ::"r"(dst), "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(0), "r"(rows[0]),
                  "r"(rows[1]), "r"(rows[2]), "r"(rows[3]), "r"(bar)
                : "memory");
        }
    };
    double acc = 0.0;
    unsigned phase = 0;
    int b = 0, pending = 0;
    long long st = wid;
    if (st < steps) { issue(st, 0); ++pending; }
    if (st + nwarps < steps) { issue(st + nwarps, 1); ++pending; }
    bool ok = true;
    for (; st < steps; st += nwarps) {
        if (!mbar_wait(bar0 + 8 * b, (phase >> b) & 1u)) {
            if (lane == 0) atomicAdd(wait_fail, 1ull);
            ok = false;
            break;
        }
        phase ^= 1u << b;
        --pending;
        const unsigned c = hash_col((unsigned long long)st * 32 + lane, seed, n);
        const double *piece = reinterpret_cast<const double *>(&slots[w][b][(lane >> 2) * 128]);
        acc += piece[(lane & 3) * 2 + (c & 1)];
        __syncwarp();
        if (lane == 0) proxy_fence();
        __syncwarp();
        if (st + 2 * nwarps < steps) { issue(st + 2 * nwarps, b); ++pending; }
        b ^= 1;
    }
    for (; !ok && pending > 0; --pending) {  // after a wait gave up: let copies in flight land
        mbar_wait(bar0 + 8 * b, (phase >> b) & 1u);
        phase ^= 1u << b;
        b ^= 1;
    }
    acc = warp_sum(acc);
    if (lane == 0) out[wid] = acc;
}

}  // namespace
}  // namespace pava

extern "C" int pava_probe_gather_tma(const double *x, long long nnz, int n,
                                     unsigned long long seed, int blocks_per_sm, double *out,
                                     unsigned long long *wait_fail, void *stream) {
    using namespace pava;
    if (!x || ((uintptr_t)x & 15) || n <= 0 || (n & 1) || nnz < 0 || blocks_per_sm <= 0 ||
        !out || !wait_fail)
        return -10;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
        return -12;
    auto encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    CUtensorMap tmap;
    const cuuint64_t dims[2] = {2, (cuuint64_t)n / 2};  // x as n / 2 rows of two doubles
    const cuuint64_t strides[1] = {16};
    const cuuint32_t box[2] = {2, 1};  // one row high, as tile::gather4 wants
    const cuuint32_t estr[2] = {1, 1};
    if (encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void *)x, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return -12;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -12;
    tma_gather_kernel<<<(unsigned)(sms * blocks_per_sm), TMA_WARPS * 32, 0,
                        (cudaStream_t)stream>>>(tmap, nnz, n, seed, out, wait_fail);
    return cudaGetLastError() == cudaSuccess ? 0 : -12;
}

extern "C" int pava_probe_floor(int mode, const double *vals, const int *cols, const double *x,
                                long long nnz, int n, unsigned long long seed,
                                int blocks_per_sm, int threads, double *out, void *stream) {
    using namespace pava;
    if (mode < 0 || mode > 3 || nnz < 0 || n <= 0 || threads <= 0 || threads % 32 != 0 ||
        threads > 1024 || blocks_per_sm <= 0 || !out)
        return -10;
    if (mode != GATHERS && (!cols || ((uintptr_t)cols & 15))) return -10;
    if ((mode == STREAMS || mode == DOT) && (!vals || ((uintptr_t)vals & 15))) return -10;
    if (mode != STREAMS && !x) return -10;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -12;
    const unsigned grid = (unsigned)(sms * blocks_per_sm);
    cudaStream_t s = (cudaStream_t)stream;
    switch (mode) {
        case STREAMS: floor_kernel<STREAMS><<<grid, threads, 0, s>>>(vals, cols, x, nnz, n, seed, out); break;
        case GATHERS: floor_kernel<GATHERS><<<grid, threads, 0, s>>>(vals, cols, x, nnz, n, seed, out); break;
        case COLGATH: floor_kernel<COLGATH><<<grid, threads, 0, s>>>(vals, cols, x, nnz, n, seed, out); break;
        default: floor_kernel<DOT><<<grid, threads, 0, s>>>(vals, cols, x, nnz, n, seed, out); break;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -12;
}

extern "C" long long pava_probe_floor_out_len(int blocks_per_sm, int threads) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -12;
    return (long long)sms * blocks_per_sm * (threads / 32);
}
