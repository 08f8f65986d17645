// The 32 engine forms the learned selector chooses between (a kernel variant and its tile
// parameters: the k = 1 candidate set of pava_autotune), their exhaustive timing, and
// selection: features (k_features.cu) -> MLP (k_mlp.cu) -> the form with the smallest
// predicted log-time that takes the matrix.  With no trained network, selection falls back to
// timing all 32.

#include <string.h>

#include <algorithm>
#include <vector>

#include "pava_internal.h"

namespace {

using namespace pava;

// Form v's format and options (the enumeration documented in pava_gpu.h).
bool form_of(int v, int &format, pava_opts &o) {
    memset(&o, 0, sizeof(o));
    if (v < 0 || v >= PAVA_NVARIANTS) return false;
    if (v < 4) {
        format = PAVA_FORMAT_CVR;
        o.steps = (v & 2) ? 128 : 64;
        o.index_mode = (v & 1) ? PAVA_INDEX_AUTO : PAVA_INDEX_I32;
    } else if (v < 12) {
        const int q = v - 4;
        format = PAVA_FORMAT_CSR5;
        o.sigma = (q & 4) ? 32 : 16;
        o.tiles_per_chunk = (q & 2) ? PAVA_TILES_WAVE : 0;
        o.index_mode = (q & 1) ? PAVA_INDEX_AUTO : PAVA_INDEX_I32;
    } else if (v < 30) {
        const int q = v - 12;
        static const int groups[3] = {1, 4, 16};
        format = PAVA_FORMAT_CSR;
        o.lanes_per_row = 1 << (q / 3);
        o.rows_per_tile = groups[q % 3] * (32 / o.lanes_per_row);
    } else {
        format = PAVA_FORMAT_SELL;
        o.index_mode = (v & 1) ? PAVA_INDEX_AUTO : PAVA_INDEX_I32;
    }
    return true;
}

}  // namespace

extern "C" {

pava_status pava_variant(int v, int *format, pava_opts *opts) {
    int f = 0;
    pava_opts o;
    if (!form_of(v, f, o)) { set_last_error("variant out of range"); return PAVA_E_INVALID_ARG; }
    if (format) *format = f;
    if (opts) *opts = o;
    return PAVA_SUCCESS;
}

int pava_variant_family(int v) {
    if (v < 0 || v >= PAVA_NVARIANTS) return -1;
    if (v < 4) return v < 2 ? 0 : 1;
    if (v < 12) return v < 8 ? 2 : 3;
    if (v < 30) return (v - 12) / 3 <= 2 ? 4 : 5;  // lanes per row <= 4 / >= 8
    return 6;
}

pava_status pava_time_variants(const pava_csr *A, int reps, double *ms, int *best) {
    if (!A || !ms) { set_last_error("NULL argument"); return PAVA_E_INVALID_ARG; }
    std::vector<pava_tune_entry> ent(PAVA_NVARIANTS);
    int n = 0, bi = -1;
    const pava_status st =
        pava_autotune(A, 1, PAVA_PREC_FP64, reps, ent.data(), PAVA_NVARIANTS, &n, &bi);
    for (int v = 0; v < PAVA_NVARIANTS; ++v) ms[v] = v < n ? ent[v].ms : -1.0;
    if (best) *best = bi;
    return st;
}

pava_status pava_select(pava_mlp *m, const pava_csr *A, int *variant, float *pred) {
    if (!m || !A || !variant) { set_last_error("NULL argument"); return PAVA_E_INVALID_ARG; }
    float f[PAVA_MLP_IN];
    pava_status st = pava_features(A, f, nullptr);
    if (st != PAVA_SUCCESS) return st;
    st = pava_mlp_set_batch(m, 1, f, nullptr, nullptr);
    static_assert(PAVA_MLP_OUT == PAVA_NVARIANTS, "one network output per form");
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
    float pred[PAVA_MLP_OUT];
    if (m && A->on_device) {
        st = pava_select(m, A, &v, pred);
    } else {  // no network (or a host CSR): exhaustive timing of the 32 forms
        double ms[PAVA_NVARIANTS];
        st = pava_time_variants(A, 3, ms, &v);
        for (int u = 0; u < PAVA_NVARIANTS; ++u) pred[u] = ms[u] > 0 ? (float)ms[u] : 3e38f;
    }
    if (st != PAVA_SUCCESS) return st;
    // the forms in order of prediction; a form that refuses the matrix (SELL padding) passes
    // the choice on to the next
    std::vector<int> order(PAVA_NVARIANTS);
    for (int u = 0; u < PAVA_NVARIANTS; ++u) order[u] = u;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return pred[a] < pred[b]; });
    for (int u : order) {
        int fmt;
        pava_opts o;
        pava_variant(u, &fmt, &o);
        st = pava_create(A, fmt, &o, stream, out);
        if (st == PAVA_SUCCESS) {
            if (variant) *variant = u;
            return st;
        }
        if (st != PAVA_E_UNSUPPORTED_PARAMS) return st;
    }
    return st;
}

}  // extern "C"
