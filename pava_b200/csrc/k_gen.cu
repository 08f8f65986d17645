// Seeded synthetic matrices generated on the device, for workloads too large to build on the
// host (the selector's training set: up to 10^7 rows and 10^8 nonzeros per matrix).
//
// Two passes: row lengths (one thread per row; block-diagonal first draws its block sizes and
// scans them), a 64-bit scan into the row pointer, then one thread per nonzero, which finds
// its row by binary search and draws its column and value.  Every draw is a counter hash of
// (seed, stream, counter), so the result does not depend on the launch shape.
//
// Columns are sorted and distinct within a row:
//   stencil   -- 2-D 5/9-point or 3-D 7/27-point neighbours on a g^d grid (natural order)
//   banded    -- L columns in the band [r - hb, r + hb] clipped to [0, n): one uniform draw
//                in each of L equal strata of the band
//   powerlaw  -- lognormal row lengths (mean, sigma, cap, share of empty rows); columns one
//                uniform draw in each of L equal strata of [0, n)
//   blockdiag -- dense diagonal blocks with sizes uniform in [bmin, bmax]
// Values are N(0,1) (Box-Muller).  Stratified columns spread like uniform draws without
// replacement but never collide, so no per-row sort or retry is needed.

#include <math.h>
#include <string.h>

#include <cub/cub.cuh>

#include "pava_internal.h"

namespace pava {

namespace {

__device__ __forceinline__ uint64_t smix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t draw(uint64_t seed, uint64_t stream, uint64_t ctr) {
    return smix(smix(seed * 0xD6E8FEB86659FD93ull + stream) ^ (ctr * 0x9E3779B97F4A7C15ull));
}
__device__ __forceinline__ double unif(uint64_t seed, uint64_t stream, uint64_t ctr) {
    return (double)(draw(seed, stream, ctr) >> 11) * 0x1.0p-53;
}
__device__ __forceinline__ double normal(uint64_t seed, uint64_t stream, uint64_t ctr) {
    const double u1 = 1.0 - unif(seed, stream, 2 * ctr);
    const double u2 = unif(seed, stream, 2 * ctr + 1);
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

constexpr uint64_t TAG_LEN = 1ull << 40;
constexpr uint64_t TAG_COL = 2ull << 40;
constexpr uint64_t TAG_VAL = 3ull << 40;
constexpr uint64_t TAG_BLK = 4ull << 40;

struct GenP {
    int family, m, n, g, dims, pts;  // g, dims, pts: stencil grid
    int hb, per_row;                 // banded
    double mu, sigma;                // powerlaw (log-space mean, sigma)
    int cap;
    double p_empty;
    int bmin, bmax;                  // blockdiag
    uint64_t seed;
};

// Stencil neighbour k (lexicographic offsets, so columns come out ascending) of row r, or -1.
__device__ __forceinline__ long long stencil_nb(const GenP &p, int r, int k) {
    const int g = p.g;
    if (p.dims == 2) {
        const int x = r % g, y = r / g;
        int dx, dy;
        if (p.pts == 5) {
            const int ox[5] = {0, -1, 0, 1, 0}, oy[5] = {-1, 0, 0, 0, 1};
            dx = ox[k]; dy = oy[k];
        } else {
            dx = k % 3 - 1; dy = k / 3 - 1;
        }
        if (x + dx < 0 || x + dx >= g || y + dy < 0 || y + dy >= g) return -1;
        return (long long)(y + dy) * g + (x + dx);
    }
    const long long gg = (long long)g * g;
    const int x = r % g, y = (r / g) % g, z = (int)(r / gg);
    int dx, dy, dz;
    if (p.pts == 7) {
        const int ox[7] = {0, 0, -1, 0, 1, 0, 0}, oy[7] = {0, -1, 0, 0, 0, 1, 0},
                  oz[7] = {-1, 0, 0, 0, 0, 0, 1};
        dx = ox[k]; dy = oy[k]; dz = oz[k];
    } else {
        dx = k % 3 - 1; dy = (k / 3) % 3 - 1; dz = k / 9 - 1;
    }
    if (x + dx < 0 || x + dx >= g || y + dy < 0 || y + dy >= g || z + dz < 0 || z + dz >= g)
        return -1;
    return (long long)(z + dz) * gg + (long long)(y + dy) * g + (x + dx);
}

__device__ __forceinline__ void band_of(const GenP &p, int r, int &lo, int &width) {
    lo = r - p.hb < 0 ? 0 : r - p.hb;
    const int hi = r + p.hb >= p.n ? p.n - 1 : r + p.hb;
    width = hi >= lo ? hi - lo + 1 : 0;
}

// Block-diagonal: block sizes for up to m / bmin + 1 blocks.
__global__ void block_size_kernel(GenP p, long long nblk, long long *__restrict__ bsz) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nblk; k += stride)
        bsz[k] = p.bmin + (long long)(draw(p.seed, TAG_BLK, (uint64_t)k) %
                                      (uint64_t)(p.bmax - p.bmin + 1));
}

__device__ __forceinline__ long long find_le(const long long *a, long long n, long long key) {
    long long lo = 0, hi = n;  // last idx with a[idx] <= key
    while (hi - lo > 1) {
        const long long mid = (lo + hi) >> 1;
        if (a[mid] <= key) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void row_len_kernel(GenP p, const long long *__restrict__ bstart, long long nblk,
                               long long *__restrict__ len) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long rr = (long long)blockIdx.x * blockDim.x + threadIdx.x; rr < p.m; rr += stride) {
        const int r = (int)rr;
        long long L = 0;
        if (p.family == PAVA_GEN_STENCIL) {
            for (int k = 0; k < p.pts; ++k) L += stencil_nb(p, r, k) >= 0;
        } else if (p.family == PAVA_GEN_BANDED) {
            int lo, w;
            band_of(p, r, lo, w);
            L = p.per_row < w ? p.per_row : w;
        } else if (p.family == PAVA_GEN_POWERLAW) {
            if (unif(p.seed, TAG_LEN + (uint64_t)r, 0) < p.p_empty) {
                L = 0;
            } else {
                const double z = normal(p.seed, TAG_LEN + (uint64_t)r, 1);
                double l = rint(exp(p.mu + p.sigma * z));
                if (l < 1) l = 1;
                if (l > p.cap) l = p.cap;
                if (l > p.n) l = p.n;
                L = (long long)l;
            }
        } else {  // blockdiag
            const long long k = find_le(bstart, nblk + 1, r);
            long long e = bstart[k + 1];
            if (e > p.m) e = p.m;
            L = e - bstart[k];
        }
        len[rr] = L;
    }
}

__global__ void rowptr_kernel(const long long *__restrict__ incl, int m, int *__restrict__ rp,
                              int *__restrict__ too_large) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r <= m; r += stride) {
        const long long v = r == 0 ? 0 : incl[r - 1];
        if (v > 2147483000LL) *too_large = 1;
        rp[r] = (int)v;
    }
}

__global__ void fill_kernel(GenP p, const int *__restrict__ rp, const long long *__restrict__ bstart,
                            long long nblk, long long nnz, int *__restrict__ ci,
                            double *__restrict__ v) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride) {
        int lo = 0, hi = p.m;  // row r: rp[r] <= j < rp[r+1]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (rp[mid] <= j) lo = mid; else hi = mid;
        }
        const int r = lo;
        const int i = (int)(j - rp[r]);
        const int L = rp[r + 1] - rp[r];
        long long c = 0;
        if (p.family == PAVA_GEN_STENCIL) {
            int seen = -1;
            for (int k = 0; k < p.pts; ++k) {
                const long long nb = stencil_nb(p, r, k);
                if (nb >= 0 && ++seen == i) { c = nb; break; }
            }
        } else if (p.family == PAVA_GEN_BANDED || p.family == PAVA_GEN_POWERLAW) {
            long long base = 0, w = p.n;
            if (p.family == PAVA_GEN_BANDED) {
                int b0, ww;
                band_of(p, r, b0, ww);
                base = b0;
                w = ww;
            }
            const long long s0 = w * i / L, s1 = w * (i + 1) / L;  // stratum [s0, s1)
            c = base + s0 + (long long)(draw(p.seed, TAG_COL + (uint64_t)r, (uint64_t)i) %
                                        (uint64_t)(s1 - s0));
        } else {
            const long long k = find_le(bstart, nblk + 1, r);
            c = bstart[k] + i;
        }
        ci[j] = (int)c;
        v[j] = normal(p.seed, TAG_VAL, (uint64_t)j);
    }
}

unsigned gridn(long long work) {
    long long b = (work + 255) / 256;
    if (b < 1) b = 1;
    if (b > 16384) b = 16384;
    return (unsigned)b;
}

}  // namespace

// Builds the generator parameters; returns false for parameters out of range.
static bool make_genp(const pava_gen_params &q, uint64_t seed, GenP &p, std::string &why) {
    memset(&p, 0, sizeof(p));
    p.family = q.family;
    p.m = q.m;
    p.n = q.n > 0 ? q.n : q.m;
    p.seed = seed;
    if (q.m < 1) { why = "m must be >= 1"; return false; }
    switch (q.family) {
        case PAVA_GEN_STENCIL: {
            p.dims = (int)q.p0;
            p.pts = (int)q.p1;
            if (!((p.dims == 2 && (p.pts == 5 || p.pts == 9)) ||
                  (p.dims == 3 && (p.pts == 7 || p.pts == 27)))) {
                why = "stencil: dims 2 with 5/9 points or dims 3 with 7/27 points";
                return false;
            }
            int g = (int)llround(pow((double)q.m, 1.0 / p.dims));
            while (g > 1 && (long long)pow((double)g, p.dims) > q.m) --g;
            if (g < 2) { why = "stencil grid smaller than 2"; return false; }
            p.g = g;
            p.m = p.n = (int)llround(pow((double)g, p.dims));
            return true;
        }
        case PAVA_GEN_BANDED:
            p.hb = (int)q.p0;
            p.per_row = (int)q.p1;
            if (p.hb < 0 || p.per_row < 1) { why = "banded: hb >= 0, per_row >= 1"; return false; }
            return true;
        case PAVA_GEN_POWERLAW: {
            const double mean = q.p0, sigma = q.p1;
            if (!(mean >= 1.0) || !(sigma >= 0.0) || q.p2 < 1 || !(q.p3 >= 0.0 && q.p3 < 1.0)) {
                why = "powerlaw: mean >= 1, sigma >= 0, cap >= 1, 0 <= p_empty < 1";
                return false;
            }
            p.sigma = sigma;
            p.mu = log(mean) - 0.5 * sigma * sigma;
            p.cap = (int)q.p2;
            p.p_empty = q.p3;
            return true;
        }
        case PAVA_GEN_BLOCKDIAG:
            p.bmin = (int)q.p0;
            p.bmax = (int)q.p1;
            if (p.bmin < 1 || p.bmax < p.bmin) { why = "blockdiag: 1 <= bmin <= bmax"; return false; }
            p.n = p.m;
            return true;
        default:
            why = "unknown generator family";
            return false;
    }
}

}  // namespace pava

extern "C" pava_status pava_gen_device(const pava_gen_params *q, uint64_t seed, void *stream,
                                       pava_csr *out) {
    using namespace pava;
    if (!q || !out) { set_last_error("NULL argument"); return PAVA_E_INVALID_ARG; }
    memset(out, 0, sizeof(*out));
    GenP p;
    std::string why;
    if (!make_genp(*q, seed, p, why)) { set_last_error(why); return PAVA_E_INVALID_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    long long nblk = 0;
    long long *bsz = nullptr, *len = nullptr;
    int *rp = nullptr, *d_flag = nullptr;
    void *tmp = nullptr;
    cudaError_t e = cudaSuccess;
    auto cleanup = [&]() {
        cudaFree(bsz); cudaFree(len); cudaFree(tmp); cudaFree(d_flag);
    };
    if (p.family == PAVA_GEN_BLOCKDIAG) {
        nblk = p.m / p.bmin + 1;
        e = cudaMalloc(&bsz, sizeof(long long) * (size_t)(nblk + 1));
        if (e == cudaSuccess) {
            block_size_kernel<<<gridn(nblk), 256, 0, s>>>(p, nblk, bsz + 1);
            e = cudaMemsetAsync(bsz, 0, sizeof(long long), s);
        }
        size_t tb = 0;
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, tb, bsz + 1, bsz + 1, nblk, s);
        if (e == cudaSuccess) e = cudaMalloc(&tmp, tb ? tb : 1);
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(tmp, tb, bsz + 1, bsz + 1, nblk, s);
        cudaFree(tmp);
        tmp = nullptr;
    }
    if (e == cudaSuccess) e = cudaMalloc(&len, sizeof(long long) * (size_t)p.m);
    if (e == cudaSuccess) e = cudaMalloc(&rp, sizeof(int) * ((size_t)p.m + 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_flag, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flag, 0, sizeof(int), s);
    if (e == cudaSuccess) {
        row_len_kernel<<<gridn(p.m), 256, 0, s>>>(p, bsz, nblk, len);
        e = cudaGetLastError();
    }
    size_t tb = 0;
    if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, tb, len, len, p.m, s);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tb ? tb : 1);
    if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(tmp, tb, len, len, p.m, s);
    if (e == cudaSuccess) {
        rowptr_kernel<<<gridn((long long)p.m + 1), 256, 0, s>>>(len, p.m, rp, d_flag);
        e = cudaGetLastError();
    }
    long long nnz = 0;
    int too_large = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nnz, len + p.m - 1, sizeof(long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&too_large, d_flag, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess || too_large) {
        cleanup();
        cudaFree(rp);
        if (too_large) { set_last_error("generated matrix exceeds 2^31 nonzeros"); return PAVA_E_TOO_LARGE; }
        set_last_error(std::string("generator: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PAVA_E_NOMEM : PAVA_E_CUDA;
    }
    int *ci = nullptr;
    double *v = nullptr;
    e = cudaMalloc(&ci, sizeof(int) * (size_t)(nnz ? nnz : 1));
    if (e == cudaSuccess) e = cudaMalloc(&v, sizeof(double) * (size_t)(nnz ? nnz : 1));
    if (e == cudaSuccess && nnz > 0) {
        fill_kernel<<<gridn(nnz), 256, 0, s>>>(p, rp, bsz, nblk, nnz, ci, v);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cleanup();
    if (e != cudaSuccess) {
        cudaFree(rp); cudaFree(ci); cudaFree(v);
        set_last_error(std::string("generator fill: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PAVA_E_NOMEM : PAVA_E_CUDA;
    }
    out->m = p.m;
    out->n = p.n;
    out->nnz = (int)nnz;
    out->row_ptr = rp;
    out->col_idx = ci;
    out->vals = v;
    out->on_device = 1;
    return PAVA_SUCCESS;
}

extern "C" pava_status pava_free_device_csr(pava_csr *A) {
    if (!A) return PAVA_SUCCESS;
    if (A->on_device) {
        cudaFree((void *)A->row_ptr);
        cudaFree((void *)A->col_idx);
        cudaFree((void *)A->vals);
    }
    memset(A, 0, sizeof(*A));
    return PAVA_SUCCESS;
}
