// Allocation-free SpMV on a caller's device CSR (pava_spmv_csr_noalloc, include/pava_gpu.h).
//
// Who needs it: callers whose device memory belongs to someone else -- a host framework that
// hands a plugin pre-allocated input and output buffers but forbids it the CUDA allocator, or
// code that runs after a fixed memory budget was committed -- cannot create a pava handle,
// because conversion allocates.  This entry point reads the caller's CSR directly and keeps
// the little scratch it needs in a fixed array compiled into the library.
//
// The kernel is the CSR5 tile kernel of k_csr5.cu without the converted layout: a warp takes
// nnz-balanced chunks of NOALLOC_G tiles of 32 lanes x NOALLOC_SIGMA elements straight from
// the CSR arrays, finds its rows by binary search in row_ptr, sums per-lane segments, combines
// the lanes with the same fixed-order suffix scan, and writes rows it does not finish to
// per-chunk carry slots.  The carry fixup of k_support.cu (unchanged) then adds those in chunk
// order.  Empty rows are zeroed by a separate pass.
//
// Scratch: one file-scope array of NOALLOC_SCRATCH_BYTES (1 MiB) per device, laid out as
// [chunk headers | head carries | tail carries] for at most NOALLOC_MAX_CHUNKS chunks.  Every
// slot a call reads is written earlier in the same call, so nothing needs clearing between
// calls; but all calls share the array, so calls that overlap on the GPU (other streams,
// other host threads) race and must be serialised by the caller.

#include <mutex>
#include <string>

#include "pava_internal.h"

namespace pava {

namespace {

constexpr int NOALLOC_SIGMA = 16;                            // elements per lane per tile
constexpr int NOALLOC_G = 8;                                 // tiles per chunk
constexpr long long NOALLOC_L = 32LL * NOALLOC_SIGMA * NOALLOC_G;  // 4096 elements per chunk
constexpr size_t NOALLOC_SCRATCH_BYTES = 1u << 20;
constexpr long long NOALLOC_MAX_CHUNKS =
    (long long)(NOALLOC_SCRATCH_BYTES / (sizeof(ChunkHdr) + 2 * sizeof(double)));  // 32768
constexpr int NOALLOC_MAX_DEVICES = 64;

// The scratch itself.  In host code this name is only a stand-in for the device symbol; the
// kernels get its device address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_setup_mutex;
void *g_scratch_addr[NOALLOC_MAX_DEVICES] = {nullptr};

// y[r] = 0 for every empty row (the tile kernel only visits rows with elements).
__global__ void zero_empty_rows_kernel(const int *__restrict__ rp, int m, double *__restrict__ y) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < m && rp[r + 1] == rp[r]) y[r] = 0.0;
}

constexpr int NA_WARPS = 8;

__global__ void __launch_bounds__(NA_WARPS * 32)
csr_tiles_noalloc_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                         const double *__restrict__ v, const double *__restrict__ x,
                         double *__restrict__ y, int m, int nnz, long long nchunks,
                         ChunkHdr *__restrict__ hdr, double *__restrict__ carry_head,
                         double *__restrict__ carry_tail, int n, unsigned long long *err) {
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * NA_WARPS;
    for (long long c = (long long)blockIdx.x * NA_WARPS + (threadIdx.x >> 5); c < nchunks;
         c += nwarps) {
        const long long s = c * NOALLOC_L;
        const long long e = s + NOALLOC_L < nnz ? s + NOALLOC_L : nnz;
        // chunk header: first / last row and whether they continue into neighbouring chunks
        const int r_first = upper_bound_m1(rp, m + 1, s);
        const int r_last = upper_bound_m1(rp, m + 1, e - 1);
        const unsigned shared = ((long long)rp[r_first] < s ? 1u : 0u) |
                                ((long long)rp[r_last + 1] > e ? 2u : 0u);
        if (lane == 0) {
            hdr[c].r_first = r_first;
            hdr[c].nrows = r_last - r_first + 1;
            hdr[c].shared = shared;
            hdr[c].aux = 0;
        }
        int carry_row = (shared & 1u) ? r_first : -1;
        double carry_val = 0.0;
        for (int tt = 0; tt < NOALLOC_G; ++tt) {
            const long long e0 = s + (long long)tt * 32 * NOALLOC_SIGMA + (long long)lane * NOALLOC_SIGMA;
            // walk this lane's elements [e0, e0 + sigma) of the chunk, tracking real rows
            int row = e0 < e ? upper_bound_m1(rp, m + 1, e0) : r_last;
            int next = rp[row + 1];
            double acc = 0.0, hpiece = 0.0;
            bool seen = false;
            for (int i = 0; i < NOALLOC_SIGMA; ++i) {
                const long long el = e0 + i;
                if (el >= e) break;  // past the matrix: nothing more in this lane
                if (el >= next) {    // a new row starts at el (skipping empty rows)
                    if (seen) y[row] = acc;
                    else { hpiece = acc; seen = true; }
                    while (rp[row + 1] <= el) ++row;
                    next = rp[row + 1];
                    acc = 0.0;
                } else if (el == e0 && (long long)rp[row] == el) {
                    seen = true;  // the lane's first element starts its row
                }
                const int col = ci[el];
                if (guard(err, col >= 0 && col < n, G_X, col)) acc = fma(v[el], x[col], acc);
            }
            if (!seen) hpiece = acc;
            const double tl = seen ? acc : 0.0;
            const unsigned sm = __ballot_sync(FULL, seen);
            const double Hs = seg_suffix(hpiece, !seen, lane);
            double Hn = __shfl_down_sync(FULL, Hs, 1);
            if (lane == 31) Hn = 0.0;
            const double H0 = __shfl_sync(FULL, Hs, 0);
            if (sm == 0) {
                carry_val += H0;  // the whole tile continues the open row
            } else {
                const int lstar = 31 - __clz(sm);
                const double own_l = tl + Hn;
                if (seen && lane != lstar) y[row] = own_l;
                const double own = __shfl_sync(FULL, own_l, lstar);
                const int own_row = __shfl_sync(FULL, row, lstar);
                if (carry_row >= 0 && lane == 0)
                    flush_row(carry_row, carry_val + H0, r_first, r_last, shared, c, y,
                              carry_head, carry_tail, m);
                carry_row = own_row;
                carry_val = own;
            }
        }
        if (carry_row >= 0 && lane == 0)
            flush_row(carry_row, carry_val, r_first, r_last, shared, c, y, carry_head,
                      carry_tail, m);
    }
}

}  // namespace

}  // namespace pava

extern "C" pava_status pava_spmv_csr_noalloc(int m, int n, int nnz, const int *row_ptr,
                                             const int *col_idx, const double *vals,
                                             const double *x, double *y, void *stream) {
    using namespace pava;
    // every error return leaves its message for pava_last_error(), as the other entry points do
    auto fail = [](pava_status st, const std::string &msg) {
        set_last_error("pava_spmv_csr_noalloc: " + msg);
        return st;
    };
    auto fail_cuda = [&](cudaError_t err, const char *where) {
        return fail(PAVA_E_CUDA, std::string(where) + ": " + cudaGetErrorString(err));
    };
    if (m < 0 || n < 0 || nnz < 0) return fail(PAVA_E_INVALID_ARG, "negative size");
    if (m == 0) return PAVA_SUCCESS;
    if (!row_ptr || !y || (nnz > 0 && (!col_idx || !vals || !x)))
        return fail(PAVA_E_INVALID_ARG, "NULL array");
    const long long nchunks = ((long long)nnz + NOALLOC_L - 1) / NOALLOC_L;
    if (nchunks > NOALLOC_MAX_CHUNKS)  // > 134,217,728 nonzeros
        return fail(PAVA_E_TOO_LARGE, "nnz " + std::to_string(nnz) +
                                          " exceeds the 134,217,728 nonzeros its fixed scratch holds");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetDevice");
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return fail(PAVA_E_INVALID_ARG, "device ordinal beyond the set-up table");
    // Set-up, once per device, on the caller's current device: the device address of the
    // scratch array.  Done by the first call on that device.
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) return fail_cuda(e, "cudaGetSymbolAddress(scratch)");
            g_scratch_addr[dev] = p;
        }
        base = g_scratch_addr[dev];
    }
    ChunkHdr *hdr = reinterpret_cast<ChunkHdr *>(base);
    double *head = reinterpret_cast<double *>(hdr + NOALLOC_MAX_CHUNKS);
    double *tail = head + NOALLOC_MAX_CHUNKS;
    cudaStream_t s = (cudaStream_t)stream;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail_cuda(e, "cudaDeviceGetAttribute");
    zero_empty_rows_kernel<<<(unsigned)(((long long)m + 255) / 256), 256, 0, s>>>(row_ptr, m, y);
    if (nchunks > 0) {
        long long blocks = (nchunks + NA_WARPS - 1) / NA_WARPS;
        if (blocks > (long long)sms * 8) blocks = (long long)sms * 8;
        csr_tiles_noalloc_kernel<<<(unsigned)blocks, NA_WARPS * 32, 0, s>>>(
            row_ptr, col_idx, vals, x, y, m, nnz, nchunks, hdr, head, tail, n, guard_word());
        // the unchanged carry fixup, pointed at the scratch: chunk c's first element is
        // c*L and a shared row R starts in chunk row_ptr[R] / L
        Handle h;
        h.m = m;
        h.nchunks = nchunks;
        h.L = NOALLOC_L;
        h.sm_count = sms;
        h.meta = hdr;
        h.meta_stride = sizeof(ChunkHdr);
        h.arp = const_cast<int *>(row_ptr);
        h.carry_head = head;
        h.carry_tail = tail;
        e = carry_fixup(h, y, s);
        h.arp = nullptr;  // the Handle owns nothing here
        h.meta = nullptr;
        h.carry_head = nullptr;
        h.carry_tail = nullptr;
        if (e != cudaSuccess) return fail_cuda(e, "carry fixup launch");
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? PAVA_SUCCESS : fail_cuda(e, "kernel launch");
}
