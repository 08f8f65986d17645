// The six engine variants the learned selector chooses between, their exhaustive timing, and
// selection: features (k_features.cu) -> MLP (k_mlp.cu) -> the variant with the smallest
// predicted log-time.  With no trained network, selection falls back to timing all six.

#include <string.h>

#include <algorithm>
#include <vector>

#include "pava_internal.h"

namespace {

using namespace pava;

struct Variant {
    int format;
    int steps, sigma, lanes_per_row;
};

constexpr Variant VARIANTS[PAVA_NVARIANTS] = {
    {PAVA_FORMAT_CVR, 64, 0, 0},  {PAVA_FORMAT_CVR, 128, 0, 0},
    {PAVA_FORMAT_CSR5, 0, 16, 0}, {PAVA_FORMAT_CSR5, 0, 32, 0},
    {PAVA_FORMAT_CSR, 0, 0, 4},   {PAVA_FORMAT_CSR, 0, 0, 32},
};

}  // namespace

extern "C" {

pava_status pava_variant(int v, int *format, pava_opts *opts) {
    if (v < 0 || v >= PAVA_NVARIANTS) { set_last_error("variant out of range"); return PAVA_E_INVALID_ARG; }
    if (format) *format = VARIANTS[v].format;
    if (opts) {
        memset(opts, 0, sizeof(*opts));
        opts->steps = VARIANTS[v].steps;
        opts->sigma = VARIANTS[v].sigma;
        opts->lanes_per_row = VARIANTS[v].lanes_per_row;
    }
    return PAVA_SUCCESS;
}

pava_status pava_time_variants(const pava_csr *A, int reps, double *ms, int *best) {
    if (!A || !ms) { set_last_error("NULL argument"); return PAVA_E_INVALID_ARG; }
    if (reps < 1) reps = 1;
    void *x = nullptr, *y = nullptr;
    cudaError_t e = cudaMalloc(&x, sizeof(double) * (size_t)(A->n ? A->n : 1));
    if (e == cudaSuccess) e = cudaMalloc(&y, sizeof(double) * (size_t)(A->m ? A->m : 1));
    if (e == cudaSuccess) e = cudaMemset(x, 0, sizeof(double) * (size_t)(A->n ? A->n : 1));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e != cudaSuccess) {
        cudaFree(x); cudaFree(y);
        if (e0) cudaEventDestroy(e0);
        set_last_error(std::string("time variants: ") + cudaGetErrorString(e));
        return PAVA_E_CUDA;
    }
    int bi = -1;
    for (int v = 0; v < PAVA_NVARIANTS; ++v) {
        ms[v] = -1.0;
        int fmt;
        pava_opts o;
        pava_variant(v, &fmt, &o);
        pava_handle *H = nullptr;
        if (pava_create(A, fmt, &o, nullptr, &H) != PAVA_SUCCESS) continue;
        pava_status st = pava_spmv(H, x, y, nullptr);
        std::vector<float> t;
        for (int r = 0; r < reps && st == PAVA_SUCCESS; ++r) {
            cudaEventRecord(e0, nullptr);
            st = pava_spmv(H, x, y, nullptr);
            cudaEventRecord(e1, nullptr);
            cudaEventSynchronize(e1);
            float f = 0.f;
            cudaEventElapsedTime(&f, e0, e1);
            t.push_back(f);
        }
        pava_destroy(H);
        if (st != PAVA_SUCCESS || t.empty()) continue;
        std::sort(t.begin(), t.end());
        ms[v] = t[t.size() / 2];
        if (bi < 0 || ms[v] < ms[bi]) bi = v;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(x);
    cudaFree(y);
    if (best) *best = bi;
    if (bi < 0) { set_last_error("no variant ran"); return PAVA_E_UNSUPPORTED_PARAMS; }
    return PAVA_SUCCESS;
}

pava_status pava_select(pava_mlp *m, const pava_csr *A, int *variant, float *pred) {
    if (!m || !A || !variant) { set_last_error("NULL argument"); return PAVA_E_INVALID_ARG; }
    float f[PAVA_MLP_IN];
    pava_status st = pava_features(A, f, nullptr);
    if (st != PAVA_SUCCESS) return st;
    st = pava_mlp_set_batch(m, 1, f, nullptr, nullptr);
    float o[PAVA_MLP_OUT];
    if (st == PAVA_SUCCESS) st = pava_mlp_forward(m, o);
    if (st != PAVA_SUCCESS) return st;
    int bi = 0;
    for (int v = 1; v < PAVA_NVARIANTS; ++v)
        if (o[v] < o[bi]) bi = v;
    *variant = bi;
    if (pred) memcpy(pred, o, sizeof(o));
    return PAVA_SUCCESS;
}

pava_status pava_create_selected(const pava_csr *A, pava_mlp *m, void *stream,
                                 pava_handle **out, int *variant) {
    if (!A || !out) { set_last_error("NULL argument"); return PAVA_E_INVALID_ARG; }
    *out = nullptr;
    int v = -1;
    pava_status st;
    if (m && A->on_device) {
        st = pava_select(m, A, &v, nullptr);
    } else {  // no network (or a host CSR): exhaustive timing of the six variants
        double ms[PAVA_NVARIANTS];
        st = pava_time_variants(A, 3, ms, &v);
    }
    if (st != PAVA_SUCCESS) return st;
    int fmt;
    pava_opts o;
    pava_variant(v, &fmt, &o);
    st = pava_create(A, fmt, &o, stream, out);
    if (st == PAVA_SUCCESS && variant) *variant = v;
    return st;
}

}  // extern "C"
