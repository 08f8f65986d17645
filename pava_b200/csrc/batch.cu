// Batches of independent matrices and the exhaustive autotuner.
//
// A batch of matrices A_0 .. A_{N-1} is held as their block-diagonal union U: rows, columns
// and nonzeros concatenated, column indices shifted by the matrix's column offset.  Then
// [y_0; ...; y_{N-1}] = U [x_0; ...; x_{N-1}] is one SpMV over the union, so the whole batch is
// one launch of any engine form, uneven sizes included; with the row-group form that launch
// is persistent (grid = resident capacity, warps take row tiles).  With k right-hand sides per
// matrix (X_i row-major n_i x k, stacked into the union's n x k X) the same union gives
// [Y_0; ...; Y_{N-1}] = U X in one persistent launch of the row-group SpMM.  A batch can record
// its SpMV or SpMM into a CUDA graph once and replay it.
//
// The autotuner converts a matrix into every candidate form and times it with CUDA events:
// it is the exhaustive search that picks tiles and lanes per row, and the measure of the
// learned selector's regret.

#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "pava_internal.h"

struct pava_batch {
    int count = 0;
    int precision = 0;
    std::vector<long long> row_off, col_off, nnz_off;  // count + 1 prefix offsets
    pava_handle *inner = nullptr;                      // the union in the chosen form
    int k = 1;                                         // right-hand sides it was tuned for
    int format = 0;
    pava_opts opts{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap_stream = nullptr;
};

namespace {

pava_status bfail(pava_status st, const std::string &msg) {
    pava::set_last_error(msg);
    return st;
}

__device__ __forceinline__ int find_seg(const long long *off, int count, long long key) {
    // last i in [0, count) with off[i] <= key
    int lo = 0, hi = count;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= key) lo = mid; else hi = mid;
    }
    return lo;
}

// Union row pointer from the matrices' own row pointers (staged back to back, m_i + 1
// entries each) and validation of each matrix's row pointer.
__global__ void union_rows_kernel(const int *__restrict__ rp_raw, const long long *row_off,
                                  const long long *nnz_off, int count, long long M,
                                  int *__restrict__ urp, int *__restrict__ err) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long R = (long long)blockIdx.x * blockDim.x + threadIdx.x; R < M; R += stride) {
        const int i = find_seg(row_off, count, R);
        const long long r = R - row_off[i];
        const int *rp = rp_raw + row_off[i] + i;
        const long long mi = row_off[i + 1] - row_off[i];
        const int a = rp[r], b = rp[r + 1];
        bool bad = b < a;
        if (r == 0 && rp[0] != 0) bad = true;
        if (r == mi - 1 && (long long)rp[mi] != nnz_off[i + 1] - nnz_off[i]) bad = true;
        if (bad) atomicAdd(err, 1);
        urp[R] = (int)(nnz_off[i] + a);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) urp[M] = (int)nnz_off[count];
}

// Shifts each matrix's columns by its column offset; counts columns outside [0, n_i).
__global__ void union_cols_kernel(int *__restrict__ ci, const long long *nnz_off,
                                  const long long *col_off, int count, long long NNZ,
                                  int *__restrict__ err) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long J = (long long)blockIdx.x * blockDim.x + threadIdx.x; J < NNZ; J += stride) {
        const int i = find_seg(nnz_off, count, J);
        const int c = ci[J];
        const long long ni = col_off[i + 1] - col_off[i];
        if (c < 0 || c >= ni) atomicAdd(err, 1);
        ci[J] = (int)(col_off[i] + c);
    }
}

unsigned grid_for(long long work) {
    long long b = (work + 255) / 256;
    if (b < 1) b = 1;
    if (b > 8192) b = 8192;
    return (unsigned)b;
}

struct UnionCSR {
    int *rp = nullptr, *ci = nullptr;
    double *v = nullptr;
    void release() {
        cudaFree(rp); cudaFree(ci); cudaFree(v);
        rp = nullptr; ci = nullptr; v = nullptr;
    }
};

pava_status build_union(int count, const pava_csr *mats, cudaStream_t s, pava_batch &b,
                        UnionCSR &u) {
    b.row_off.assign(count + 1, 0);
    b.col_off.assign(count + 1, 0);
    b.nnz_off.assign(count + 1, 0);
    for (int i = 0; i < count; ++i) {
        const pava_csr &A = mats[i];
        if (A.m < 0 || A.n < 0 || A.nnz < 0) return bfail(PAVA_E_INVALID_ARG, "negative size");
        if (!A.row_ptr || (A.nnz > 0 && (!A.col_idx || !A.vals)))
            return bfail(PAVA_E_INVALID_ARG, "NULL CSR array in batch matrix " + std::to_string(i));
        if (A.m == 0 && A.nnz > 0)
            return bfail(PAVA_E_INVALID_CSR, "batch matrix " + std::to_string(i) +
                                                 " has nonzeros but no rows");
        b.row_off[i + 1] = b.row_off[i] + A.m;
        b.col_off[i + 1] = b.col_off[i] + A.n;
        b.nnz_off[i + 1] = b.nnz_off[i] + A.nnz;
    }
    const long long M = b.row_off[count], N = b.col_off[count], NNZ = b.nnz_off[count];
    if (M >= INT32_MAX - 1 || N >= INT32_MAX - 1 || NNZ >= INT32_MAX - 64)
        return bfail(PAVA_E_TOO_LARGE, "batch union exceeds the int32 index space");
    int *rp_raw = nullptr, *d_err = nullptr;
    long long *d_off = nullptr;
    cudaError_t e = cudaMalloc(&u.rp, sizeof(int) * (size_t)(M + 1));
    if (e == cudaSuccess) e = cudaMalloc(&u.ci, sizeof(int) * (size_t)(NNZ ? NNZ : 1));
    if (e == cudaSuccess) e = cudaMalloc(&u.v, sizeof(double) * (size_t)(NNZ ? NNZ : 1));
    if (e == cudaSuccess) e = cudaMalloc(&rp_raw, sizeof(int) * (size_t)(M + count));
    if (e == cudaSuccess) e = cudaMalloc(&d_off, sizeof(long long) * 3 * (size_t)(count + 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), s);
    for (int i = 0; i < count && e == cudaSuccess; ++i) {
        const pava_csr &A = mats[i];
        const cudaMemcpyKind kind = A.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        e = cudaMemcpyAsync(rp_raw + b.row_off[i] + i, A.row_ptr, sizeof(int) * ((size_t)A.m + 1),
                            kind, s);
        if (e == cudaSuccess && A.nnz)
            e = cudaMemcpyAsync(u.ci + b.nnz_off[i], A.col_idx, sizeof(int) * (size_t)A.nnz, kind, s);
        if (e == cudaSuccess && A.nnz)
            e = cudaMemcpyAsync(u.v + b.nnz_off[i], A.vals, sizeof(double) * (size_t)A.nnz, kind, s);
    }
    const size_t ob = sizeof(long long) * (size_t)(count + 1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_off, b.row_off.data(), ob, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_off + (count + 1), b.col_off.data(), ob, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_off + 2 * (count + 1), b.nnz_off.data(), ob, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        union_rows_kernel<<<grid_for(M), 256, 0, s>>>(rp_raw, d_off, d_off + 2 * (count + 1),
                                                      count, M, u.rp, d_err);
        union_cols_kernel<<<grid_for(NNZ), 256, 0, s>>>(u.ci, d_off + 2 * (count + 1),
                                                        d_off + (count + 1), count, NNZ, d_err);
        e = cudaGetLastError();
    }
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(rp_raw);
    cudaFree(d_off);
    cudaFree(d_err);
    if (e != cudaSuccess) {
        u.release();
        return bfail(e == cudaErrorMemoryAllocation ? PAVA_E_NOMEM : PAVA_E_CUDA,
                     std::string("batch union: ") + cudaGetErrorString(e));
    }
    if (herr) {
        u.release();
        return bfail(PAVA_E_INVALID_CSR, "batch matrix with a bad row pointer or column (" +
                                             std::to_string(herr) + " violations)");
    }
    return PAVA_SUCCESS;
}

// Built-in candidate forms for k right-hand sides: for k = 1 the 32 forms of pava_variant in
// their order (the selector's space); for k > 1 the row-group shapes (at most 72 for k <= 128)
// and the SELL SpMM shapes (lanes per row x column form, at most 4).
std::vector<std::pair<int, pava_opts>> candidates(int k, int precision) {
    std::vector<std::pair<int, pava_opts>> c;
    auto base = [&]() {
        pava_opts o;
        memset(&o, 0, sizeof(o));
        o.precision = precision;
        return o;
    };
    if (k == 1) {
        for (int v = 0; v < PAVA_NVARIANTS; ++v) {
            int f = 0;
            pava_opts o;
            pava_variant(v, &f, &o);
            o.precision = precision;
            c.push_back({f, o});
        }
        return c;
    }
    const int kpls[3] = {1, 2, 4};
    for (int kpl : kpls) {
        int kc = 1;
        while (kc * kpl < k) kc <<= 1;
        if (kc > 32) continue;
        if (kpl > 1 && kc * (kpl / 2) >= k) continue;  // a smaller kpl covers k already
        for (int gl = kc; gl <= 32; gl <<= 1)
            for (int groups : {1, 4, 16}) {
                pava_opts o = base();
                o.lanes_per_row = gl;
                o.col_lanes = kc;
                o.cols_per_lane = kpl;
                o.rows_per_tile = groups * (32 / gl);
                c.push_back({PAVA_FORMAT_CSR, o});
            }
        if (k > 1)  // X windows in shared memory: CTA tiles of 128 or 256 rows
            for (int gl = kc; gl <= 32; gl <<= 1)
                for (int tr : {128, 256}) {
                    pava_opts o = base();
                    o.lanes_per_row = gl;
                    o.col_lanes = kc;
                    o.cols_per_lane = kpl;
                    o.x_window = 1;
                    o.rows_per_tile = tr;  // a multiple of 8 * 32 / gl for every gl >= 2
                    c.push_back({PAVA_FORMAT_CSR, o});
                }
    }
    // SELL: 4 (k <= 32) or 8 lanes per row, 32-bit columns or 16-bit offsets where they reach
    // (16 lanes per row, an option of pava_create, was never faster on the banded, stencil and
    // batch matrices)
    for (int g : {4, 8}) {
        if (pava::sell_spmm_lanes(g, k) == 0) continue;
        for (int idx : {PAVA_INDEX_I32, PAVA_INDEX_AUTO}) {
            pava_opts o = base();
            o.lanes_per_row = g;
            o.index_mode = idx;
            c.push_back({PAVA_FORMAT_SELL, o});
        }
    }
    return c;
}

}  // namespace

extern "C" {

pava_status pava_autotune(const pava_csr *A, int k, int precision, int reps,
                          pava_tune_entry *entries, int max_entries, int *n_entries, int *best) {
    if (!A || !n_entries || !best) return bfail(PAVA_E_INVALID_ARG, "NULL argument");
    if (k < 1 || k > 128) return bfail(PAVA_E_INVALID_ARG, "k must be in [1, 128]");
    if (precision != PAVA_PREC_FP64 && precision != PAVA_PREC_FP32C)
        return bfail(PAVA_E_UNSUPPORTED_VALUE_TYPE, "unknown precision");
    if (reps < 1) reps = 1;
    *n_entries = 0;
    *best = -1;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return bfail(PAVA_E_CUDA, "no usable CUDA device");
    const std::vector<std::pair<int, pava_opts>> cand = candidates(k, precision);
    // CSR5 forms whose wave-balanced tile count equals the default count are the same form:
    // timed once, the twin copies the result
    auto csr5_tiles = [&](const pava_opts &o) {
        const long long tiles = (long long)A->nnz / (32LL * o.sigma), warps = 24LL * sms;
        if (o.tiles_per_chunk == PAVA_TILES_WAVE) return pava::csr5_wave_tiles(tiles, warps);
        return o.tiles_per_chunk ? o.tiles_per_chunk : pava::csr5_default_tiles(tiles, warps);
    };
    const size_t sx = precision == PAVA_PREC_FP32C ? 4 : 8;
    void *X = nullptr, *Y = nullptr;
    cudaError_t e = cudaMalloc(&X, sx * (size_t)(A->n ? A->n : 1) * k);
    if (e == cudaSuccess) e = cudaMalloc(&Y, sizeof(double) * (size_t)(A->m ? A->m : 1) * k);
    if (e == cudaSuccess) e = cudaMemset(X, 0, sx * (size_t)(A->n ? A->n : 1) * k);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e != cudaSuccess) {
        cudaFree(X); cudaFree(Y);
        if (e0) cudaEventDestroy(e0);
        return bfail(PAVA_E_CUDA, std::string("autotune setup: ") + cudaGetErrorString(e));
    }
    double best_ms = 1e300;
    int n = 0;
    for (size_t ci = 0; ci < cand.size() && n < max_entries; ++ci) {
        pava_tune_entry &t = entries[n++];
        t.format = cand[ci].first;
        t.opts = cand[ci].second;
        t.ms = -1.0;
        if (t.format == PAVA_FORMAT_CSR5 && t.opts.tiles_per_chunk == PAVA_TILES_WAVE && n >= 3) {
            // forms 4 + 4s + 2w + a: the default-tiles twin of a wave form is two entries back
            const pava_tune_entry &tw = entries[n - 3];
            if (tw.format == PAVA_FORMAT_CSR5 && tw.opts.tiles_per_chunk == 0 &&
                tw.opts.sigma == t.opts.sigma && tw.opts.index_mode == t.opts.index_mode &&
                csr5_tiles(tw.opts) == csr5_tiles(t.opts)) {
                t.ms = tw.ms;
                t.status = tw.status;
                continue;
            }
        }
        pava_handle *H = nullptr;
        t.status = pava_create(A, t.format, &t.opts, nullptr, &H);
        if (t.status != PAVA_SUCCESS) continue;
        auto run = [&]() {
            return k == 1 ? pava_spmv(H, X, Y, nullptr) : pava_spmm(H, k, X, k, Y, k, nullptr);
        };
        pava_status st = run();
        if (st == PAVA_SUCCESS) st = run();
        std::vector<float> ms;
        for (int r = 0; r < reps && st == PAVA_SUCCESS; ++r) {
            cudaEventRecord(e0, nullptr);
            st = run();
            cudaEventRecord(e1, nullptr);
            cudaEventSynchronize(e1);
            float v = 0.f;
            cudaEventElapsedTime(&v, e0, e1);
            ms.push_back(v);
        }
        pava_destroy(H);
        t.status = st;
        if (st != PAVA_SUCCESS || ms.empty()) continue;
        std::sort(ms.begin(), ms.end());
        t.ms = ms[ms.size() / 2];
        if (t.ms < best_ms) {
            best_ms = t.ms;
            *best = n - 1;
        }
    }
    *n_entries = n;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(X);
    cudaFree(Y);
    if (*best < 0) return bfail(PAVA_E_UNSUPPORTED_PARAMS, "no candidate form ran");
    return PAVA_SUCCESS;
}

pava_status pava_batch_create_spmm(int count, const pava_csr *mats, int k, int format,
                                   const pava_opts *opts, void *stream, pava_batch **out) {
    if (!out) return bfail(PAVA_E_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (count < 1 || !mats) return bfail(PAVA_E_INVALID_ARG, "empty batch");
    if (k < 1 || k > 128) return bfail(PAVA_E_INVALID_ARG, "k must be in [1, 128]");
    if (k > 1 && format >= 0 && format != PAVA_FORMAT_CSR && format != PAVA_FORMAT_SELL)
        return bfail(PAVA_E_UNKNOWN_FORMAT,
                     "k > 1 right-hand sides need the CSR row-group or the SELL form");
    if (k > 1 && format == PAVA_FORMAT_SELL &&
        pava::sell_spmm_lanes(opts ? opts->lanes_per_row : 0, k) == 0)
        return bfail(PAVA_E_UNSUPPORTED_PARAMS, "SELL SpMM takes k <= 64 (k <= 32 with 4 lanes)");
    pava_batch *b = new (std::nothrow) pava_batch();
    if (!b) return bfail(PAVA_E_NOMEM, "host allocation failed");
    b->count = count;
    b->k = k;
    pava_opts o;
    memset(&o, 0, sizeof(o));
    if (opts) o = *opts;
    b->precision = o.precision;
    cudaStream_t s = (cudaStream_t)stream;
    UnionCSR u;
    pava_status st = build_union(count, mats, s, *b, u);
    if (st != PAVA_SUCCESS) { delete b; return st; }
    pava_csr U{(int)b->row_off[count], (int)b->col_off[count], (int)b->nnz_off[count], u.rp,
               u.ci, u.v, 1};
    if (format < 0) {  // autotune over the built-in candidates for k right-hand sides
        std::vector<pava_tune_entry> ent(128);
        int ne = 0, bi = -1;
        st = pava_autotune(&U, k, o.precision, 5, ent.data(), (int)ent.size(), &ne, &bi);
        if (st != PAVA_SUCCESS) { u.release(); delete b; return st; }
        format = ent[bi].format;
        o = ent[bi].opts;
    }
    b->format = format;
    b->opts = o;
    st = pava_create(&U, format, &o, stream, &b->inner);
    u.release();
    if (st != PAVA_SUCCESS) {
        delete b;
        return st;
    }
    *out = b;
    return PAVA_SUCCESS;
}

pava_status pava_batch_create(int count, const pava_csr *mats, int format, const pava_opts *opts,
                              void *stream, pava_batch **out) {
    return pava_batch_create_spmm(count, mats, 1, format, opts, stream, out);
}

pava_status pava_batch_layout(const pava_batch *b, long long *x_offsets, long long *y_offsets,
                              long long *nnz_offsets) {
    if (!b) return bfail(PAVA_E_INVALID_ARG, "batch is NULL");
    const size_t n = (size_t)b->count + 1;
    if (x_offsets) memcpy(x_offsets, b->col_off.data(), n * sizeof(long long));
    if (y_offsets) memcpy(y_offsets, b->row_off.data(), n * sizeof(long long));
    if (nnz_offsets) memcpy(nnz_offsets, b->nnz_off.data(), n * sizeof(long long));
    return PAVA_SUCCESS;
}

pava_status pava_batch_get(const pava_batch *b, int *format, pava_opts *opts, pava_info *info) {
    if (!b) return bfail(PAVA_E_INVALID_ARG, "batch is NULL");
    if (format) *format = b->format;
    if (opts) *opts = b->opts;
    if (info) return pava_get_info(b->inner, info);
    return PAVA_SUCCESS;
}

pava_status pava_batch_spmv(pava_batch *b, const void *x, void *y, void *stream) {
    if (!b) return bfail(PAVA_E_INVALID_ARG, "batch is NULL");
    return pava_spmv(b->inner, x, y, stream);
}

pava_status pava_batch_spmm(pava_batch *b, int k, const void *X, long long ldx, void *Y,
                            long long ldy, void *stream) {
    if (!b) return bfail(PAVA_E_INVALID_ARG, "batch is NULL");
    return pava_spmm(b->inner, k, X, ldx, Y, ldy, stream);
}

}  // extern "C"

namespace {

// Records one product on the batch's capture stream into the batch's graph (replacing any
// earlier one); `run` issues the launches on the stream it is given.
template <typename F>
pava_status capture_into(pava_batch *b, F run) {
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    cudaError_t e = cudaSuccess;
    if (!b->cap_stream) e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess)
        return bfail(PAVA_E_CUDA, std::string("begin capture: ") + cudaGetErrorString(e));
    pava_status st = run(b->cap_stream);
    e = cudaStreamEndCapture(b->cap_stream, &b->graph);
    if (st != PAVA_SUCCESS) {
        if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
        return st;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess)
        return bfail(PAVA_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    return PAVA_SUCCESS;
}

}  // namespace

extern "C" {

pava_status pava_batch_capture(pava_batch *b, const void *x, void *y) {
    if (!b) return bfail(PAVA_E_INVALID_ARG, "batch is NULL");
    return capture_into(b, [&](cudaStream_t cs) { return pava_spmv(b->inner, x, y, cs); });
}

pava_status pava_batch_capture_spmm(pava_batch *b, int k, const void *X, long long ldx, void *Y,
                                    long long ldy) {
    if (!b) return bfail(PAVA_E_INVALID_ARG, "batch is NULL");
    return capture_into(
        b, [&](cudaStream_t cs) { return pava_spmm(b->inner, k, X, ldx, Y, ldy, cs); });
}

pava_status pava_batch_replay(pava_batch *b, void *stream) {
    if (!b) return bfail(PAVA_E_INVALID_ARG, "batch is NULL");
    if (!b->exec) return bfail(PAVA_E_NOT_CONVERTED, "no captured graph: call pava_batch_capture");
    cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) return bfail(PAVA_E_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
    return PAVA_SUCCESS;
}

pava_status pava_batch_destroy(pava_batch *b) {
    if (!b) return PAVA_SUCCESS;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    pava_destroy(b->inner);
    delete b;
    return PAVA_SUCCESS;
}

}  // extern "C"
