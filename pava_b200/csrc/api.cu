// C ABI of the engine (include/pava_gpu.h): handles, conversion, SpMV dispatch, and the
// reference-shaped drop-ins conduct_cvr_gpu / conduct_csr5_gpu.

#include <stdio.h>
#include <string.h>

#include <atomic>
#include <climits>
#include <mutex>
#include <string>

#include "pava_internal.h"

// Pipeline of the asynchronous host-buffer entry point: two staging slots, one stream each for
// copies in, SpMVs and copies out, and per-slot events that order the reuse of a slot.
struct HostPipe {
    bool ready = false;
    cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
    cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_comp[2] = {nullptr, nullptr},
                ev_out[2] = {nullptr, nullptr};
    void *x[2] = {nullptr, nullptr}, *y[2] = {nullptr, nullptr};
    unsigned long long calls = 0;
};

struct pava_handle {
    pava::Handle h;
    void *x_dev = nullptr;  // buffers of the host-buffer entry point
    void *y_dev = nullptr;
    HostPipe pipe;
};

namespace {

void free_pipe(HostPipe &p) {
    if (p.out) cudaStreamSynchronize(p.out);
    for (int k = 0; k < 2; ++k) {
        if (p.ev_in[k]) cudaEventDestroy(p.ev_in[k]);
        if (p.ev_comp[k]) cudaEventDestroy(p.ev_comp[k]);
        if (p.ev_out[k]) cudaEventDestroy(p.ev_out[k]);
        cudaFree(p.x[k]);
        cudaFree(p.y[k]);
    }
    if (p.in) cudaStreamDestroy(p.in);
    if (p.comp) cudaStreamDestroy(p.comp);
    if (p.out) cudaStreamDestroy(p.out);
    p = HostPipe();
}

cudaError_t make_pipe(HostPipe &p, size_t sx, size_t sy) {
    cudaError_t e = cudaStreamCreateWithFlags(&p.in, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p.comp, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p.out, cudaStreamNonBlocking);
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        e = cudaEventCreateWithFlags(&p.ev_in[k], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p.ev_comp[k], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p.ev_out[k], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&p.x[k], sx);
        if (e == cudaSuccess) e = cudaMalloc(&p.y[k], sy);
    }
    if (e != cudaSuccess) free_pipe(p);
    else p.ready = true;
    return e;
}

}  // namespace

namespace {

thread_local std::string g_last_error;

pava_status fail(pava_status st, const std::string &msg) {
    g_last_error = msg;
    return st;
}

pava_status fail_cuda(cudaError_t e, const char *where) {
    std::string msg = std::string(where) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return fail(PAVA_E_NOMEM, msg);
    return fail(PAVA_E_CUDA, msg);
}

#define PAVA_CUDA(call, where)                               \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return fail_cuda(e_, where);  \
    } while (0)

// Bytes of device memory one handle may hold (0: no limit), pava_set_device_memory_limit.
std::atomic<unsigned long long> g_mem_limit{0};

// A handle's device allocation: counted in *acc and refused, as an allocation failure, when it
// would take the handle past the memory limit.
cudaError_t budget_malloc(void **p, size_t bytes, size_t *acc) {
    *p = nullptr;
    if (bytes == 0) bytes = 1;
    const unsigned long long lim = g_mem_limit.load();
    if (lim && acc && (unsigned long long)*acc + bytes > lim) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess && acc) *acc += bytes;
    return e;
}

template <typename T>
cudaError_t dalloc(T **p, size_t count, size_t *acc) {
    return budget_malloc((void **)p, sizeof(T) * (count ? count : 1), acc);
}

void free_handle_buffers(pava::Handle &h) {
    cudaFree(h.arp);
    cudaFree(h.vals);
    cudaFree(h.cols);
    cudaFree(h.flags);
    cudaFree(h.meta);
    cudaFree(h.tile_ptr);
    cudaFree(h.colbase);
    cudaFree(h.carry_head);
    cudaFree(h.carry_tail);
    cudaFree(h.rp);
    cudaFree(h.ci);
    cudaFree(h.v);
    h.arp = nullptr; h.vals = nullptr; h.cols = nullptr; h.flags = nullptr; h.meta = nullptr;
    h.tile_ptr = nullptr; h.colbase = nullptr; h.carry_head = nullptr; h.carry_tail = nullptr;
    h.rp = nullptr; h.ci = nullptr; h.v = nullptr;
}

int auto_lanes_per_row(int m, int nnz) {
    const double mean = m > 0 ? (double)nnz / m : 0.0;
    if (mean <= 2) return 1;
    if (mean <= 4) return 2;
    if (mean <= 8) return 4;
    if (mean <= 16) return 8;
    if (mean <= 32) return 16;
    return 32;
}

size_t value_bytes(int precision) { return precision == PAVA_PREC_FP32C ? 4 : 8; }

bool pow2_le32(int v) { return v == 1 || v == 2 || v == 4 || v == 8 || v == 16 || v == 32; }

int pow2_ceil(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// The row-group shape of a CSR handle for k right-hand sides: the handle's options where
// given, otherwise derived from k and the mean row length.  Returns false (with a message)
// when the given options cannot serve k.
bool resolve_group_shape(const pava::Handle &h, int k, pava::Handle &out, std::string &why) {
    out = h;
    int kpl = h.cols_per_lane, kc = h.col_lanes;
    if (kpl == 0 && kc == 0) {
        kpl = k <= 32 ? 1 : (k <= 64 ? 2 : 4);
        kc = pow2_ceil((k + kpl - 1) / kpl);
    } else if (kpl == 0) {
        kpl = (long long)kc >= k ? 1 : ((long long)kc * 2 >= k ? 2 : 4);
    } else if (kc == 0) {
        kc = pow2_ceil((k + kpl - 1) / kpl);
    }
    if (kc > 32 || (long long)kc * kpl < k) {
        why = "col_lanes * cols_per_lane must cover k (col_lanes <= 32, cols_per_lane <= 4)";
        return false;
    }
    int gl = h.lanes_per_row;
    if (gl == 0) gl = k == 1 ? auto_lanes_per_row(h.m, h.nnz) : kc;
    if (gl < kc) gl = h.lanes_per_row == 0 ? kc : gl;
    if (!pow2_le32(gl) || gl < kc) {
        why = "lanes_per_row must be a power of two <= 32 and >= col_lanes";
        return false;
    }
    const int gpw = 32 / gl;
    const int unit = h.x_window ? 8 * gpw : gpw;  // rows one pass of a warp / of a CTA covers
    int tr = h.rows_per_tile ? h.rows_per_tile : 4 * unit;
    if (tr % unit != 0) {
        why = h.x_window ? "rows_per_tile must be a multiple of 8 * 32 / lanes_per_row with x_window"
                         : "rows_per_tile must be a multiple of 32 / lanes_per_row";
        return false;
    }
    out.lanes_per_row = gl;
    out.col_lanes = kc;
    out.cols_per_lane = kpl;
    out.rows_per_tile = tr;
    return true;
}

// Builds the augmented row pointer and sizes the chunked element space (CVR, CSR5).
pava_status plan_chunks(pava::Handle &h, const int *rp, cudaStream_t s) {
    PAVA_CUDA(dalloc(&h.arp, (size_t)h.m + 2, &h.device_bytes), "cudaMalloc(arp)");
    int *d_nempty = nullptr;
    PAVA_CUDA(cudaMallocAsync(&d_nempty, sizeof(int), s), "cudaMallocAsync");
    cudaError_t e = pava::build_augmented_rowptr(rp, h.m, 0, h.arp, d_nempty, s);
    int nempty = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nempty, d_nempty, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(d_nempty, s);
    if (e != cudaSuccess) return fail_cuda(e, "augmented row pointer");
    h.n_empty = nempty;
    h.n_aug = (long long)h.nnz + nempty;
    h.nchunks = (h.n_aug + h.L - 1) / h.L;
    const long long padded = h.nchunks * h.L;
    if (padded >= (long long)INT_MAX - 64)
        return fail(PAVA_E_TOO_LARGE, "matrix exceeds the int32 element space after padding");
    const int pt = (int)padded;
    PAVA_CUDA(cudaMemcpyAsync(h.arp + h.m + 1, &pt, sizeof(int), cudaMemcpyHostToDevice, s),
              "cudaMemcpyAsync(arp)");
    PAVA_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    return PAVA_SUCCESS;
}

pava_status convert(pava::Handle &h, const int *rp, const int *ci, const double *v,
                    cudaStream_t s) {
    const size_t sv = value_bytes(h.precision);
    const size_t si = h.index_mode == PAVA_INDEX_DELTA16 ? 2 : 4;
    if (h.format == PAVA_FORMAT_CVR || h.format == PAVA_FORMAT_CSR5) {
        pava_status st = plan_chunks(h, rp, s);
        if (st != PAVA_SUCCESS) return st;
        const size_t padded = (size_t)(h.nchunks * h.L);
        PAVA_CUDA(budget_malloc(&h.vals, sv * (padded ? padded : 1), &h.device_bytes),
                  "cudaMalloc(vals)");
        PAVA_CUDA(budget_malloc(&h.cols, si * (padded ? padded : 1), &h.device_bytes),
                  "cudaMalloc(cols)");
        PAVA_CUDA(dalloc(&h.carry_head, (size_t)h.nchunks, &h.device_bytes), "cudaMalloc(carry)");
        PAVA_CUDA(dalloc(&h.carry_tail, (size_t)h.nchunks, &h.device_bytes), "cudaMalloc(carry)");
        if (h.index_mode == PAVA_INDEX_DELTA16) {
            PAVA_CUDA(dalloc(&h.colbase, (size_t)h.nchunks, &h.device_bytes), "cudaMalloc(colbase)");
            PAVA_CUDA(pava::chunk_colbase(h, rp, ci, s), "chunk column bases");
        }
        int *d_ovf = nullptr;
        PAVA_CUDA(cudaMallocAsync(&d_ovf, sizeof(int), s), "cudaMallocAsync");
        cudaError_t e = cudaMemsetAsync(d_ovf, 0, sizeof(int), s);
        if (h.format == PAVA_FORMAT_CVR) {
            if (e == cudaSuccess) e = dalloc(&h.flags, (size_t)h.nchunks * h.S, &h.device_bytes);
            h.meta_stride = sizeof(pava::CvrMeta);
            if (e == cudaSuccess)
                e = dalloc((pava::CvrMeta **)&h.meta, (size_t)h.nchunks, &h.device_bytes);
            if (e == cudaSuccess) e = pava::cvr_convert(h, rp, ci, v, d_ovf, s);
        } else {
            h.ntiles = h.nchunks * h.G;
            if (e == cudaSuccess) e = dalloc(&h.flags, (size_t)h.ntiles * 32, &h.device_bytes);
            if (e == cudaSuccess) e = dalloc(&h.tile_ptr, (size_t)h.ntiles, &h.device_bytes);
            h.meta_stride = sizeof(pava::ChunkHdr);
            if (e == cudaSuccess)
                e = dalloc((pava::ChunkHdr **)&h.meta, (size_t)h.nchunks, &h.device_bytes);
            if (e == cudaSuccess) e = pava::csr5_convert(h, rp, ci, v, d_ovf, s);
        }
        int ovf = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&ovf, d_ovf, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFreeAsync(d_ovf, s);
        if (e != cudaSuccess) return fail_cuda(e, "conversion");
        h.d16_overflow = ovf ? 1 : 0;
        if (ovf)
            return fail(PAVA_E_UNSUPPORTED_PARAMS,
                        "16-bit column offsets: a chunk's columns span more than 65534");
    } else if (h.format == PAVA_FORMAT_SELL) {  // slices of 32 rows, padded, block layout
        h.nchunks = ((long long)h.m + 31) / 32;
        h.L = 32;
        h.meta_stride = sizeof(pava::SellSlice);
        PAVA_CUDA(dalloc((pava::SellSlice **)&h.meta, (size_t)h.nchunks, &h.device_bytes),
                  "cudaMalloc(slices)");
        int *d_off = nullptr, *d_tot = nullptr, *d_ovf = nullptr;
        int total_blk = 0, ovf = 0;
        cudaError_t e = cudaMallocAsync(&d_off, sizeof(int) * (size_t)(h.nchunks + 1), s);
        if (e == cudaSuccess) e = cudaMallocAsync(&d_tot, sizeof(int), s);
        if (e == cudaSuccess) e = cudaMallocAsync(&d_ovf, sizeof(int), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_ovf, 0, sizeof(int), s);
        if (e == cudaSuccess && h.nchunks > 0) e = pava::sell_plan(h, rp, ci, d_off, d_tot, s);
        if (e == cudaSuccess && h.nchunks > 0)
            e = cudaMemcpyAsync(&total_blk, d_tot, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        const long long padded = (long long)total_blk * 128;
        pava_status st = PAVA_SUCCESS;
        if (e != cudaSuccess) {
            st = fail_cuda(e, "SELL plan");
        } else if (padded > 2LL * h.nnz + 128LL * h.nchunks) {
            st = fail(PAVA_E_UNSUPPORTED_PARAMS,
                      "SELL: padding the slices would more than double the stored elements (" +
                          std::to_string(padded) + " for " + std::to_string(h.nnz) + " nonzeros)");
        } else if (padded >= (long long)INT_MAX - 64) {
            st = fail(PAVA_E_TOO_LARGE, "SELL: padded elements exceed the int32 element space");
        } else {
            h.n_aug = padded;
            e = budget_malloc(&h.vals, sv * (size_t)(padded ? padded : 1), &h.device_bytes);
            if (e == cudaSuccess)
                e = budget_malloc(&h.cols, si * (size_t)(padded ? padded : 1), &h.device_bytes);
            if (e == cudaSuccess && h.nchunks > 0) e = pava::sell_fill(h, rp, ci, v, d_off, d_ovf, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(&ovf, d_ovf, sizeof(int), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) st = fail_cuda(e, "SELL conversion");
        }
        cudaFreeAsync(d_off, s);
        cudaFreeAsync(d_tot, s);
        cudaFreeAsync(d_ovf, s);
        if (st != PAVA_SUCCESS) return st;
        h.d16_overflow = ovf ? 1 : 0;
        if (ovf)
            return fail(PAVA_E_UNSUPPORTED_PARAMS,
                        "16-bit column offsets: a slice's columns span more than 65534");
    } else {  // plain CSR: private copies (values narrowed to float for FP32C)
        PAVA_CUDA(dalloc(&h.rp, (size_t)h.m + 1, &h.device_bytes), "cudaMalloc(rp)");
        PAVA_CUDA(dalloc(&h.ci, (size_t)h.nnz, &h.device_bytes), "cudaMalloc(ci)");
        const size_t nv = (size_t)(h.nnz ? h.nnz : 1);
        PAVA_CUDA(budget_malloc(&h.v, sv * nv, &h.device_bytes), "cudaMalloc(v)");
        PAVA_CUDA(cudaMemcpyAsync(h.rp, rp, sizeof(int) * ((size_t)h.m + 1),
                                  cudaMemcpyDeviceToDevice, s), "copy rp");
        if (h.nnz > 0) {
            PAVA_CUDA(cudaMemcpyAsync(h.ci, ci, sizeof(int) * (size_t)h.nnz,
                                      cudaMemcpyDeviceToDevice, s), "copy ci");
            if (h.precision == PAVA_PREC_FP32C)
                PAVA_CUDA(pava::narrow_to_float(v, (float *)h.v, h.nnz, s), "narrow values");
            else
                PAVA_CUDA(cudaMemcpyAsync(h.v, v, sizeof(double) * (size_t)h.nnz,
                                          cudaMemcpyDeviceToDevice, s), "copy v");
        }
        h.nchunks = h.m;
        h.L = 0;
    }
    return PAVA_SUCCESS;
}

}  // namespace

#ifdef PAVA_BOUNDS_CHECK
// The bounds-check error word: [0] failed tests, [1] site of the first, [2] its index.
__device__ unsigned long long g_guard_word[3];
namespace {
constexpr int GUARD_MAX_DEVICES = 64;
void *g_guard_addr[GUARD_MAX_DEVICES] = {};
std::mutex g_guard_mutex;
}  // namespace
#endif

// The bounded-wait word: [0] waits that gave up, [1] site of the first + 1 (SELL: its slice).
__device__ unsigned long long g_wait_word[2];
namespace {
constexpr int WAIT_MAX_DEVICES = 64;
void *g_wait_addr[WAIT_MAX_DEVICES] = {};
std::mutex g_wait_mutex;
}  // namespace

namespace pava {
void set_last_error(const std::string &msg) { g_last_error = msg; }

unsigned long long *wait_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= WAIT_MAX_DEVICES) return nullptr;
    std::lock_guard<std::mutex> lock(g_wait_mutex);
    if (!g_wait_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_wait_word) != cudaSuccess) return nullptr;
        g_wait_addr[dev] = p;
    }
    return (unsigned long long *)g_wait_addr[dev];
}

unsigned long long *guard_word() {
#ifdef PAVA_BOUNDS_CHECK
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= GUARD_MAX_DEVICES) return nullptr;
    std::lock_guard<std::mutex> lock(g_guard_mutex);
    if (!g_guard_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_guard_word) != cudaSuccess) return nullptr;
        g_guard_addr[dev] = p;
    }
    return (unsigned long long *)g_guard_addr[dev];
#else
    return nullptr;
#endif
}
}  // namespace pava

extern "C" {

int pava_bounds_checked(void) {
#ifdef PAVA_BOUNDS_CHECK
    return 1;
#else
    return 0;
#endif
}

pava_status pava_bounds_report(unsigned long long *out3, int clear) {
#ifdef PAVA_BOUNDS_CHECK
    unsigned long long *w = pava::guard_word();
    if (!w) return fail(PAVA_E_CUDA, "bounds-check error word unavailable");
    unsigned long long h[3] = {0, 0, 0};
    PAVA_CUDA(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    PAVA_CUDA(cudaMemcpy(h, w, sizeof(h), cudaMemcpyDeviceToHost), "read bounds-check word");
    if (clear) PAVA_CUDA(cudaMemset(w, 0, sizeof(h)), "clear bounds-check word");
    if (out3) memcpy(out3, h, sizeof(h));
    return PAVA_SUCCESS;
#else
    (void)clear;
    if (out3) memset(out3, 0, 3 * sizeof(unsigned long long));
    return fail(PAVA_E_UNSUPPORTED_PARAMS, "not a bounds-checked build (PAVA_BOUNDS_CHECK)");
#endif
}

pava_status pava_wait_report(unsigned long long *out2, int clear) {
    unsigned long long *w = pava::wait_word();
    if (!w) return fail(PAVA_E_CUDA, "bounded-wait word unavailable");
    unsigned long long h[2] = {0, 0};
    PAVA_CUDA(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    PAVA_CUDA(cudaMemcpy(h, w, sizeof(h), cudaMemcpyDeviceToHost), "read bounded-wait word");
    if (clear) PAVA_CUDA(cudaMemset(w, 0, sizeof(h)), "clear bounded-wait word");
    if (out2) memcpy(out2, h, sizeof(h));
    return h[0] ? PAVA_E_TIMEOUT : PAVA_SUCCESS;
}

pava_status pava_set_device_memory_limit(unsigned long long bytes) {
    g_mem_limit.store(bytes);
    return PAVA_SUCCESS;
}

unsigned long long pava_get_device_memory_limit(void) { return g_mem_limit.load(); }

pava_status pava_init(int device) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(PAVA_E_CUDA, std::string("no usable CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= count) return fail(PAVA_E_INVALID_ARG, "device out of range");
    PAVA_CUDA(cudaSetDevice(device), "cudaSetDevice");
    return PAVA_SUCCESS;
}

const char *pava_last_error(void) { return g_last_error.c_str(); }

const char *pava_status_string(int st) {
    switch (st) {
        case PAVA_SUCCESS: return "success";
        case PAVA_E_UNKNOWN_FORMAT: return "unknown format";
        case PAVA_E_UNSUPPORTED_PARAMS: return "unsupported tile parameters";
        case PAVA_E_CONVERT_FAILED: return "conversion failed";
        case PAVA_E_NOT_CONVERTED: return "spmv on a matrix that is not converted";
        case PAVA_E_UNSUPPORTED_VALUE_TYPE: return "unsupported value type";
        case PAVA_E_INVALID_ARG: return "invalid argument";
        case PAVA_E_INVALID_CSR: return "invalid CSR";
        case PAVA_E_CUDA: return "CUDA error";
        case PAVA_E_NOMEM: return "out of device memory";
        case PAVA_E_TIMEOUT: return "device wait timed out";
        case PAVA_E_TOO_LARGE: return "matrix too large";
        default: return "unknown status";
    }
}

pava_status pava_create(const pava_csr *A, int format, const pava_opts *opts, void *stream,
                        pava_handle **out) {
    if (!out) return fail(PAVA_E_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (!A) return fail(PAVA_E_INVALID_ARG, "matrix is NULL");
    if (format != PAVA_FORMAT_CSR && format != PAVA_FORMAT_CSR5 && format != PAVA_FORMAT_CVR &&
        format != PAVA_FORMAT_SELL)
        return fail(PAVA_E_UNKNOWN_FORMAT, "unknown format");
    if (A->m < 0 || A->n < 0 || A->nnz < 0) return fail(PAVA_E_INVALID_ARG, "negative size");
    if (!A->row_ptr || (A->nnz > 0 && (!A->col_idx || !A->vals)))
        return fail(PAVA_E_INVALID_ARG, "NULL CSR array");
    pava_opts o;
    memset(&o, 0, sizeof(o));
    if (opts) o = *opts;
    // sizes that cannot fit the int32 element space of the chunked forms, however few rows are
    // empty (the largest chunk is 32 x 32 x 64 elements): refused before any array is read
    if (format != PAVA_FORMAT_CSR && (long long)A->nnz + 65536 >= (long long)INT_MAX - 64)
        return fail(PAVA_E_TOO_LARGE, "nnz " + std::to_string(A->nnz) +
                                          " leaves no room for chunk padding in the int32 "
                                          "element space");
    if (A->m == INT_MAX)  // m + 1 row pointers and the padding row must be indexable
        return fail(PAVA_E_TOO_LARGE, "m must be below 2^31 - 1");
    if (o.precision != PAVA_PREC_FP64 && o.precision != PAVA_PREC_FP32C)
        return fail(PAVA_E_UNSUPPORTED_VALUE_TYPE, "unknown precision");
    if (o.index_mode != PAVA_INDEX_I32 && o.index_mode != PAVA_INDEX_DELTA16 &&
        o.index_mode != PAVA_INDEX_AUTO)
        return fail(PAVA_E_UNSUPPORTED_PARAMS, "unknown index mode");
    if (format == PAVA_FORMAT_CSR && o.index_mode == PAVA_INDEX_AUTO) o.index_mode = PAVA_INDEX_I32;
    if (format == PAVA_FORMAT_CSR && o.index_mode != PAVA_INDEX_I32)
        return fail(PAVA_E_UNSUPPORTED_PARAMS, "the plain CSR form takes 32-bit columns");
    const bool auto_index = o.index_mode == PAVA_INDEX_AUTO;
    if (auto_index) o.index_mode = PAVA_INDEX_DELTA16;  // tried first

    pava_handle *H = new (std::nothrow) pava_handle();
    if (!H) return fail(PAVA_E_NOMEM, "host allocation failed");
    pava::Handle &h = H->h;
    h.format = format;
    h.precision = o.precision;
    h.index_mode = o.index_mode;
    h.m = A->m;
    h.n = A->n;
    h.nnz = A->nnz;
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&h.sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (ce != cudaSuccess) { delete H; return fail_cuda(ce, "no usable CUDA device"); }
    h.device = dev;
    // default chunk sizes: the larger forms unless that leaves fewer than ~24 warp chunks per
    // SM (small matrices), where shorter chunks keep every SM busy
    const long long want_chunks = 24LL * h.sm_count;
    if (format == PAVA_FORMAT_CVR) {
        h.S = o.steps ? o.steps : ((long long)h.nnz / (32 * 64) < want_chunks ? 32 : 64);
        if (h.S != 32 && h.S != 64 && h.S != 128) {
            delete H;
            return fail(PAVA_E_UNSUPPORTED_PARAMS, "CVR steps must be 32, 64 or 128");
        }
        h.L = 32LL * h.S;
    } else if (format == PAVA_FORMAT_CSR5) {
        h.sigma = o.sigma ? o.sigma : 16;
        if (o.tiles_per_chunk == PAVA_TILES_WAVE) {  // fill the last wave of warps best
            h.G = pava::csr5_wave_tiles((long long)h.nnz / (32LL * h.sigma), want_chunks);
        } else if (o.tiles_per_chunk) {
            h.G = o.tiles_per_chunk;
        } else {  // 4 tiles per chunk, fewer for small matrices
            h.G = pava::csr5_default_tiles((long long)h.nnz / (32LL * h.sigma), want_chunks);
        }
        if (!(h.sigma == 8 || h.sigma == 12 || h.sigma == 16 || h.sigma == 24 || h.sigma == 32) ||
            h.G < 1 || h.G > 64) {
            delete H;
            return fail(PAVA_E_UNSUPPORTED_PARAMS, "CSR5 sigma must be 8/12/16/24/32, tiles 1..64");
        }
        h.L = 32LL * h.sigma * h.G;
    } else if (format == PAVA_FORMAT_SELL) {
        // a slice is 32 rows, its block 4 steps; lanes_per_row: the SpMM's lanes per row
        if (!(o.lanes_per_row == 0 || o.lanes_per_row == 4 || o.lanes_per_row == 8 ||
              o.lanes_per_row == 16)) {
            delete H;
            return fail(PAVA_E_UNSUPPORTED_PARAMS, "SELL lanes_per_row must be 0, 4, 8 or 16");
        }
        h.lanes_per_row = o.lanes_per_row;
    } else {
        // 0 = derive per call (resolve_group_shape)
        h.lanes_per_row = o.lanes_per_row;
        h.col_lanes = o.col_lanes;
        h.cols_per_lane = o.cols_per_lane;
        h.rows_per_tile = o.rows_per_tile;
        h.x_window = o.x_window ? 1 : 0;
        std::string why;
        pava::Handle probe;
        if ((o.lanes_per_row && !pow2_le32(o.lanes_per_row)) ||
            (o.col_lanes && !pow2_le32(o.col_lanes)) ||
            !(o.cols_per_lane == 0 || o.cols_per_lane == 1 || o.cols_per_lane == 2 ||
              o.cols_per_lane == 4) ||
            o.rows_per_tile < 0 || o.rows_per_tile > (1 << 20) ||
            !resolve_group_shape(h, 1, probe, why)) {
            delete H;
            return fail(PAVA_E_UNSUPPORTED_PARAMS,
                        why.empty() ? "CSR group shape: lanes_per_row / col_lanes powers of two "
                                      "<= 32, cols_per_lane 1, 2 or 4"
                                    : why);
        }
    }

    // inputs on the device
    const int *rp = A->row_ptr, *ci = A->col_idx;
    const double *v = A->vals;
    int *t_rp = nullptr, *t_ci = nullptr;
    double *t_v = nullptr;
    pava_status st = PAVA_SUCCESS;
    auto cleanup_tmp = [&]() {
        cudaFree(t_rp); cudaFree(t_ci); cudaFree(t_v);
    };
    if (!A->on_device) {
        ce = cudaMalloc(&t_rp, sizeof(int) * ((size_t)h.m + 1));
        if (ce == cudaSuccess) ce = cudaMalloc(&t_ci, sizeof(int) * (size_t)(h.nnz ? h.nnz : 1));
        if (ce == cudaSuccess) ce = cudaMalloc(&t_v, sizeof(double) * (size_t)(h.nnz ? h.nnz : 1));
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(t_rp, rp, sizeof(int) * ((size_t)h.m + 1), cudaMemcpyHostToDevice, s);
        if (ce == cudaSuccess && h.nnz)
            ce = cudaMemcpyAsync(t_ci, ci, sizeof(int) * (size_t)h.nnz, cudaMemcpyHostToDevice, s);
        if (ce == cudaSuccess && h.nnz)
            ce = cudaMemcpyAsync(t_v, v, sizeof(double) * (size_t)h.nnz, cudaMemcpyHostToDevice, s);
        if (ce != cudaSuccess) { cleanup_tmp(); delete H; return fail_cuda(ce, "copying the CSR to the device"); }
        rp = t_rp; ci = t_ci; v = t_v;
    }
    // validation
    {
        int *d_err = nullptr;
        int herr = 0;
        ce = cudaMallocAsync(&d_err, sizeof(int), s);
        if (ce == cudaSuccess) ce = pava::launch_validate(rp, ci, h.m, h.n, h.nnz, d_err, s);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
        cudaFreeAsync(d_err, s);
        if (ce != cudaSuccess) { cleanup_tmp(); delete H; return fail_cuda(ce, "CSR validation"); }
        if (herr) {
            cleanup_tmp();
            delete H;
            return fail(PAVA_E_INVALID_CSR, "row_ptr not monotone, row_ptr[0]/row_ptr[m] wrong, or column out of range (" +
                                                std::to_string(herr) + " violations)");
        }
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    st = convert(h, rp, ci, v, s);
    if (st == PAVA_E_UNSUPPORTED_PARAMS && auto_index && h.d16_overflow) {
        // a column does not fit 16 bits: convert again with 32-bit columns
        free_handle_buffers(h);
        h.device_bytes = 0;
        h.index_mode = PAVA_INDEX_I32;
        st = convert(h, rp, ci, v, s);
    }
    if (st == PAVA_SUCCESS) {
        cudaEventRecord(e1, s);
        ce = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
        if (ce != cudaSuccess) st = fail_cuda(ce, "conversion");
        h.convert_ms = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cleanup_tmp();
    if (st != PAVA_SUCCESS) {
        free_handle_buffers(h);
        delete H;
        return st;
    }
    *out = H;
    return PAVA_SUCCESS;
}

pava_status pava_spmv_stage(pava_handle *H, const void *x, void *y, void *stream, int stage) {
    if (!H) return fail(PAVA_E_INVALID_ARG, "handle is NULL");
    if (stage < 0 || stage > 2) return fail(PAVA_E_INVALID_ARG, "stage must be 0, 1 or 2");
    pava::Handle &h = H->h;
    if (h.m == 0) return PAVA_SUCCESS;
    if (!x || !y) return fail(PAVA_E_INVALID_ARG, "x or y is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    const bool main_k = stage != 2, fix_k = stage != 1;
    if (h.format == PAVA_FORMAT_CVR) {
        if (main_k) e = pava::cvr_spmv(h, x, y, s);
        if (e == cudaSuccess && fix_k) e = pava::carry_fixup(h, y, s);
    } else if (h.format == PAVA_FORMAT_CSR5) {
        if (main_k) e = pava::csr5_spmv(h, x, y, s);
        if (e == cudaSuccess && fix_k) e = pava::carry_fixup(h, y, s);
    } else if (h.format == PAVA_FORMAT_SELL) {  // one pass: every row ends in its own lane
        if (main_k) e = pava::sell_spmv(h, x, y, s);
    } else {
        if (main_k) {
            pava::Handle g;
            std::string why;
            if (!resolve_group_shape(h, 1, g, why)) return fail(PAVA_E_UNSUPPORTED_PARAMS, why);
            e = pava::csr_spmv(g, x, y, s);
        }
    }
    if (e != cudaSuccess) return fail_cuda(e, "spmv launch");
    return PAVA_SUCCESS;
}

pava_status pava_spmm(pava_handle *H, int k, const void *X, long long ldx, void *Y,
                      long long ldy, void *stream) {
    if (!H) return fail(PAVA_E_INVALID_ARG, "handle is NULL");
    pava::Handle &h = H->h;
    if (h.format != PAVA_FORMAT_CSR && h.format != PAVA_FORMAT_SELL)
        return fail(PAVA_E_UNKNOWN_FORMAT, "pava_spmm needs a CSR or SELL handle");
    if (k < 1 || k > 128) return fail(PAVA_E_INVALID_ARG, "k must be in [1, 128]");
    if (ldx < k || ldy < k) return fail(PAVA_E_INVALID_ARG, "ldx and ldy must be >= k");
    if (h.m == 0) return PAVA_SUCCESS;
    if (!X || !Y) return fail(PAVA_E_INVALID_ARG, "X or Y is NULL");
    if (h.format == PAVA_FORMAT_SELL) {
        if (pava::sell_spmm_lanes(h.lanes_per_row, k) == 0)
            return fail(PAVA_E_UNSUPPORTED_PARAMS,
                        "SELL SpMM takes k <= 64 (k <= 32 with 4 lanes per row)");
        const cudaError_t e = pava::sell_spmm(h, X, ldx, Y, ldy, k, (cudaStream_t)stream);
        if (e != cudaSuccess) return fail_cuda(e, "spmm launch");
        return PAVA_SUCCESS;
    }
    pava::Handle g;
    std::string why;
    if (!resolve_group_shape(h, k, g, why)) return fail(PAVA_E_UNSUPPORTED_PARAMS, why);
    cudaError_t e = pava::csr_spmm(g, X, ldx, Y, ldy, k, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "spmm launch");
    return PAVA_SUCCESS;
}

pava_status pava_spmv(pava_handle *H, const void *x, void *y, void *stream) {
    return pava_spmv_stage(H, x, y, stream, 0);
}

pava_status pava_spmv_host(pava_handle *H, const void *x_host, void *y_host, void *stream) {
    if (!H) return fail(PAVA_E_INVALID_ARG, "handle is NULL");
    pava::Handle &h = H->h;
    if (!x_host || !y_host) return fail(PAVA_E_INVALID_ARG, "x or y is NULL");
    const size_t sx = value_bytes(h.precision) * (size_t)(h.n ? h.n : 1);
    const size_t sy = sizeof(double) * (size_t)(h.m ? h.m : 1);
    if (!H->x_dev) PAVA_CUDA(cudaMalloc(&H->x_dev, sx), "cudaMalloc(x)");
    if (!H->y_dev) PAVA_CUDA(cudaMalloc(&H->y_dev, sy), "cudaMalloc(y)");
    cudaStream_t s = (cudaStream_t)stream;
    PAVA_CUDA(cudaMemcpyAsync(H->x_dev, x_host, sx, cudaMemcpyHostToDevice, s), "copy x");
    pava_status st = pava_spmv(H, H->x_dev, H->y_dev, stream);
    if (st != PAVA_SUCCESS) return st;
    PAVA_CUDA(cudaMemcpyAsync(y_host, H->y_dev, sy, cudaMemcpyDeviceToHost, s), "copy y");
    PAVA_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    return PAVA_SUCCESS;
}

pava_status pava_spmv_host_async(pava_handle *H, const void *x_host, void *y_host,
                                 void *stream) {
    if (!H) return fail(PAVA_E_INVALID_ARG, "handle is NULL");
    pava::Handle &h = H->h;
    if (!x_host || !y_host) return fail(PAVA_E_INVALID_ARG, "x or y is NULL");
    const size_t sx = value_bytes(h.precision) * (size_t)(h.n ? h.n : 1);
    const size_t sy = sizeof(double) * (size_t)(h.m ? h.m : 1);
    HostPipe &p = H->pipe;
    if (!p.ready) PAVA_CUDA(make_pipe(p, sx, sy), "host pipeline set-up");
    const int k = (int)(p.calls & 1);
    cudaStream_t s = (cudaStream_t)stream;
    // copy in: after the SpMV that last read this slot (not after the caller's stream, which
    // waits for earlier calls' copies out: x_host must be ready when the call is made)
    if (p.calls >= 2) PAVA_CUDA(cudaStreamWaitEvent(p.in, p.ev_comp[k], 0), "cudaStreamWaitEvent");
    PAVA_CUDA(cudaMemcpyAsync(p.x[k], x_host, sx, cudaMemcpyHostToDevice, p.in), "copy x");
    PAVA_CUDA(cudaEventRecord(p.ev_in[k], p.in), "cudaEventRecord");
    // SpMV: after its x arrived and after the copy-out that last read this slot's y
    PAVA_CUDA(cudaStreamWaitEvent(p.comp, p.ev_in[k], 0), "cudaStreamWaitEvent");
    if (p.calls >= 2) PAVA_CUDA(cudaStreamWaitEvent(p.comp, p.ev_out[k], 0), "cudaStreamWaitEvent");
    pava_status st = pava_spmv(H, p.x[k], p.y[k], p.comp);
    if (st != PAVA_SUCCESS) return st;
    PAVA_CUDA(cudaEventRecord(p.ev_comp[k], p.comp), "cudaEventRecord");
    // copy out, and the caller's stream waits for it
    PAVA_CUDA(cudaStreamWaitEvent(p.out, p.ev_comp[k], 0), "cudaStreamWaitEvent");
    PAVA_CUDA(cudaMemcpyAsync(y_host, p.y[k], sy, cudaMemcpyDeviceToHost, p.out), "copy y");
    PAVA_CUDA(cudaEventRecord(p.ev_out[k], p.out), "cudaEventRecord");
    PAVA_CUDA(cudaStreamWaitEvent(s, p.ev_out[k], 0), "cudaStreamWaitEvent");
    ++p.calls;
    return PAVA_SUCCESS;
}

pava_status pava_spmv_host_wait(pava_handle *H) {
    if (!H) return fail(PAVA_E_INVALID_ARG, "handle is NULL");
    if (H->pipe.ready) PAVA_CUDA(cudaStreamSynchronize(H->pipe.out), "cudaStreamSynchronize");
    return PAVA_SUCCESS;
}

pava_status pava_get_info(const pava_handle *H, pava_info *out) {
    if (!H || !out) return fail(PAVA_E_INVALID_ARG, "NULL argument");
    const pava::Handle &h = H->h;
    memset(out, 0, sizeof(*out));
    out->format = h.format;
    out->precision = h.precision;
    out->index_mode = h.index_mode;
    out->m = h.m;
    out->n = h.n;
    out->nnz = h.nnz;
    out->n_empty = h.n_empty;
    out->chunks = h.nchunks;
    out->elems_per_chunk = h.L;
    out->convert_ms = h.convert_ms;
    out->device_bytes = h.device_bytes;
    const double sv = (double)value_bytes(h.precision);
    const double si = h.index_mode == PAVA_INDEX_DELTA16 ? 2.0 : 4.0;
    out->alg_bytes = (double)h.nnz * (sv + si) + 4.0 * ((double)h.m + 1) + (double)h.n * sv +
                     (double)h.m * 8.0;
    const double xy = (double)h.n * sv + (double)h.m * 8.0;
    if (h.format == PAVA_FORMAT_CVR)
        out->format_bytes = (double)h.nchunks * h.L * (sv + si) + (double)h.nchunks * h.S * 4.0 +
                            (double)h.nchunks * sizeof(pava::CvrMeta) + xy;
    else if (h.format == PAVA_FORMAT_CSR5)
        out->format_bytes = (double)h.nchunks * h.L * (sv + si) + (double)h.ntiles * (32 * 4 + 4) +
                            (double)h.nchunks * sizeof(pava::ChunkHdr) + xy;
    else if (h.format == PAVA_FORMAT_SELL)  // padded slices and their descriptors
        out->format_bytes = (double)h.n_aug * (sv + si) +
                            (double)h.nchunks * sizeof(pava::SellSlice) + xy;
    else
        out->format_bytes = (double)h.nnz * (sv + si) + 4.0 * ((double)h.m + 1) + xy;
    return PAVA_SUCCESS;
}

pava_status pava_destroy(pava_handle *H) {
    if (!H) return PAVA_SUCCESS;
    free_pipe(H->pipe);
    free_handle_buffers(H->h);
    cudaFree(H->x_dev);
    cudaFree(H->y_dev);
    delete H;
    return PAVA_SUCCESS;
}

}  // extern "C"

// ---- conduct_cvr_gpu / conduct_csr5_gpu --------------------------------------------------

namespace {

int conduct_gpu(int format, int m, int n, int nnz, const int *rp, const int *ci,
                const double *v, const double *x, double *y, const char *name, int iters,
                const pava_opts *opts, pava_run_record *rec) {
    pava_csr A{m, n, nnz, rp, ci, v, 0};
    pava_handle *H = nullptr;
    pava_opts o;
    memset(&o, 0, sizeof(o));
    if (opts) o = *opts;
    else o.index_mode = PAVA_INDEX_AUTO;  // 16-bit column offsets where they fit: same results
    if (rec) {
        memset(rec, 0, sizeof(*rec));
        rec->status = PAVA_E_INVALID_ARG;
        rec->convert_s = rec->exec_s = -1.0;
    }
    const char *fname = format == PAVA_FORMAT_CVR    ? "CVR"
                        : format == PAVA_FORMAT_CSR5 ? "CSR5"
                        : format == PAVA_FORMAT_SELL ? "SELL"
                                                     : "CSR";
    int st = pava_create(&A, format, &o, nullptr, &H);
    if (st != PAVA_SUCCESS) {
        printf(" Performance %s %s %d %f %f \n", name ? name : "", fname, 0, -1.0, -1.0);
        if (rec) rec->status = st;
        return st;
    }
    // the checked first call, then the timed calls (cvr/cvr.h:2108-2112; csr5/csr5.h:149-153)
    st = pava_spmv_host(H, x, y, nullptr);
    double exec_s = -1.0;
    if (st == PAVA_SUCCESS && iters > 0) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, nullptr);
        for (int i = 0; i < iters && st == PAVA_SUCCESS; ++i)
            st = pava_spmv(H, H->x_dev, H->y_dev, nullptr);
        cudaEventRecord(b, nullptr);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        exec_s = ms * 1e-3 / iters;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    printf(" Performance %s %s %d %f %f \n", name ? name : "", fname, H->h.sm_count,
           H->h.convert_ms * 1e-3, exec_s);
    fflush(stdout);
    if (rec) {
        const pava::Handle &h = H->h;
        pava_info inf;
        pava_get_info(H, &inf);
        rec->status = st;
        rec->format = h.format;
        rec->precision = h.precision;
        rec->index_mode = h.index_mode;
        rec->steps = h.S;
        rec->sigma = h.sigma;
        rec->tiles_per_chunk = h.G;
        rec->lanes_per_row = h.lanes_per_row;
        rec->sm_count = h.sm_count;
        rec->iterations = iters;
        rec->chunks = h.nchunks;
        rec->convert_s = h.convert_ms * 1e-3;
        rec->exec_s = exec_s;
        rec->alg_bytes = inf.alg_bytes;
        rec->format_bytes = inf.format_bytes;
    }
    pava_destroy(H);
    return st;
}

}  // namespace

extern "C" int pava_conduct(int format, const pava_csr *A, const double *x, double *y,
                            const char *name, int iterations, const pava_opts *opts,
                            pava_run_record *rec) {
    if (!A || A->on_device || !x || !y) {
        g_last_error = "pava_conduct: host CSR, x and y required";
        return PAVA_E_INVALID_ARG;
    }
    return conduct_gpu(format, A->m, A->n, A->nnz, A->row_ptr, A->col_idx, A->vals, x, y, name,
                       iterations, opts, rec);
}

extern "C" int conduct_cvr_gpu(int numRows, int numCols, int nItems_raw, int *h_rowDelimiters,
                               int *h_cols, double *h_val, double *h_vec, double *refOut,
                               int alpha, char *matrixName, int numIterations) {
    (void)alpha;
    return conduct_gpu(PAVA_FORMAT_CVR, numRows, numCols, nItems_raw, h_rowDelimiters, h_cols,
                       h_val, h_vec, refOut, matrixName, numIterations, nullptr, nullptr);
}

extern "C" int conduct_csr5_gpu(int m, int n, int nnzA, int *csrRowPtrA, int *csrColIdxA,
                                double *csrValA, double *x, double *y, double alpha,
                                char *matrixName, int numIterations) {
    (void)alpha;
    return conduct_gpu(PAVA_FORMAT_CSR5, m, n, nnzA, csrRowPtrA, csrColIdxA, csrValA, x, y,
                       matrixName, numIterations, nullptr, nullptr);
}
