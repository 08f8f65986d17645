// The learned form selector's network: an MLP 12 -> 64 -> 64 -> 6 (ReLU, FP32) that predicts
// the log-time of each of the six engine variants from a matrix's structural features
// (k_features.cu), trained on the GPU by the kernels below (forward, backward, Adam).
//
// Parameters, one flat float array of 5,382 entries:
//   W1[64][12] @0   b1[64] @768   W2[64][64] @832   b2[64] @4928   W3[6][64] @4992   b3[6] @5376
// Loss: masked mean squared error over the six outputs (a variant that failed on a matrix
// has mask 0).  Every reduction runs in a fixed order (one thread owns one sum), so a
// training run gives the same bits every time.

#include <math.h>
#include <string.h>

#include <vector>

#include "pava_internal.h"

namespace pava {

namespace {

constexpr int IN = PAVA_MLP_IN, HID = PAVA_MLP_HIDDEN, OUT = PAVA_MLP_OUT;
constexpr int OW1 = 0, OB1 = OW1 + HID * IN, OW2 = OB1 + HID, OB2 = OW2 + HID * HID,
              OW3 = OB2 + HID, OB3 = OW3 + OUT * HID, NP = OB3 + OUT;
static_assert(NP == PAVA_MLP_NPARAM, "parameter count");

// One block of HID threads per sample.  Stores pre-activations Z1, Z2 and outputs O.
__global__ void __launch_bounds__(HID)
forward_kernel(const float *__restrict__ P, const float *__restrict__ X, int B,
               float *__restrict__ Z1, float *__restrict__ Z2, float *__restrict__ O) {
    __shared__ float xs[IN], h1[HID], h2[HID];
    const int b = blockIdx.x, j = threadIdx.x;
    if (b >= B) return;
    if (j < IN) xs[j] = X[(long long)b * IN + j];
    __syncthreads();
    float z = P[OB1 + j];
    for (int i = 0; i < IN; ++i) z = fmaf(P[OW1 + j * IN + i], xs[i], z);
    Z1[(long long)b * HID + j] = z;
    h1[j] = z > 0.f ? z : 0.f;
    __syncthreads();
    z = P[OB2 + j];
    for (int k = 0; k < HID; ++k) z = fmaf(P[OW2 + j * HID + k], h1[k], z);
    Z2[(long long)b * HID + j] = z;
    h2[j] = z > 0.f ? z : 0.f;
    __syncthreads();
    if (j < OUT) {
        float o = P[OB3 + j];
        for (int k = 0; k < HID; ++k) o = fmaf(P[OW3 + j * HID + k], h2[k], o);
        O[(long long)b * OUT + j] = o;
    }
}

// Per-sample backward: dO = 2 mask (O - T) / count, then dZ2 and dZ1 through the ReLUs.
__global__ void __launch_bounds__(HID)
backward_kernel(const float *__restrict__ P, int B, const float *__restrict__ Z1,
                const float *__restrict__ Z2, const float *__restrict__ O,
                const float *__restrict__ T, const float *__restrict__ Mk, float inv_count,
                float *__restrict__ dO, float *__restrict__ dZ1, float *__restrict__ dZ2) {
    __shared__ float go[OUT], g2[HID];
    const int b = blockIdx.x, j = threadIdx.x;
    if (b >= B) return;
    if (j < OUT) {
        const long long q = (long long)b * OUT + j;
        const float g = 2.f * Mk[q] * (O[q] - T[q]) * inv_count;
        go[j] = g;
        dO[q] = g;
    }
    __syncthreads();
    float s = 0.f;
    for (int t = 0; t < OUT; ++t) s = fmaf(go[t], P[OW3 + t * HID + j], s);
    const float d2 = Z2[(long long)b * HID + j] > 0.f ? s : 0.f;
    g2[j] = d2;
    dZ2[(long long)b * HID + j] = d2;
    __syncthreads();
    s = 0.f;
    for (int k = 0; k < HID; ++k) s = fmaf(g2[k], P[OW2 + k * HID + j], s);
    dZ1[(long long)b * HID + j] = Z1[(long long)b * HID + j] > 0.f ? s : 0.f;
}

// One thread per parameter: its gradient summed over the batch in sample order.
__global__ void grad_kernel(const float *__restrict__ X, int B, const float *__restrict__ Z1,
                            const float *__restrict__ Z2, const float *__restrict__ dO,
                            const float *__restrict__ dZ1, const float *__restrict__ dZ2,
                            float *__restrict__ G) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    float s = 0.f;
    if (p < OB1) {
        const int j = (p - OW1) / IN, i = (p - OW1) % IN;
        for (int b = 0; b < B; ++b) s = fmaf(dZ1[(long long)b * HID + j], X[(long long)b * IN + i], s);
    } else if (p < OW2) {
        const int j = p - OB1;
        for (int b = 0; b < B; ++b) s += dZ1[(long long)b * HID + j];
    } else if (p < OB2) {
        const int j = (p - OW2) / HID, k = (p - OW2) % HID;
        for (int b = 0; b < B; ++b) {
            const float h = Z1[(long long)b * HID + k];
            s = fmaf(dZ2[(long long)b * HID + j], h > 0.f ? h : 0.f, s);
        }
    } else if (p < OW3) {
        const int j = p - OB2;
        for (int b = 0; b < B; ++b) s += dZ2[(long long)b * HID + j];
    } else if (p < OB3) {
        const int t = (p - OW3) / HID, k = (p - OW3) % HID;
        for (int b = 0; b < B; ++b) {
            const float h = Z2[(long long)b * HID + k];
            s = fmaf(dO[(long long)b * OUT + t], h > 0.f ? h : 0.f, s);
        }
    } else {
        const int t = p - OB3;
        for (int b = 0; b < B; ++b) s += dO[(long long)b * OUT + t];
    }
    G[p] = s;
}

// Masked mean squared error, one block: strided partial sums, then a fixed tree.
__global__ void __launch_bounds__(256)
loss_kernel(const float *__restrict__ O, const float *__restrict__ T,
            const float *__restrict__ Mk, long long n, float inv_count, float *__restrict__ out) {
    __shared__ float part[256];
    float s = 0.f;
    for (long long q = threadIdx.x; q < n; q += 256) {
        const float d = O[q] - T[q];
        s = fmaf(Mk[q] * d, d, s);
    }
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0] * inv_count;
}

__global__ void adam_kernel(float *__restrict__ P, const float *__restrict__ G,
                            float *__restrict__ Mm, float *__restrict__ Vv, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    const float g = G[p];
    const float m = b1 * Mm[p] + (1.f - b1) * g;
    const float v = b2 * Vv[p] + (1.f - b2) * g * g;
    Mm[p] = m;
    Vv[p] = v;
    P[p] -= lr * (m * c1) / (sqrtf(v * c2) + eps);
}

// (x - mean) / std per feature.
__global__ void normalize_kernel(float *__restrict__ X, int B, const float *__restrict__ mu,
                                 const float *__restrict__ sd) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)B * IN) return;
    const int i = (int)(q % IN);
    X[q] = (X[q] - mu[i]) / sd[i];
}

// splitmix64 -> uniform in [-1, 1)
uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace
}  // namespace pava

struct pava_mlp {
    float *P = nullptr, *G = nullptr, *Mm = nullptr, *Vv = nullptr;  // params, grad, Adam
    float *mu = nullptr, *sd = nullptr;                              // feature normalisation
    int B = 0, cap = 0;
    float *X = nullptr, *T = nullptr, *Mk = nullptr;                 // current batch
    float *Z1 = nullptr, *Z2 = nullptr, *O = nullptr, *dO = nullptr, *dZ1 = nullptr,
          *dZ2 = nullptr, *loss = nullptr;
    float inv_count = 0.f;
    int step = 0;
};

namespace {

using namespace pava;

pava_status mfail(cudaError_t e, const char *where) {
    set_last_error(std::string(where) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? PAVA_E_NOMEM : PAVA_E_CUDA;
}

void free_batch(pava_mlp *m) {
    float **bufs[] = {&m->X, &m->T, &m->Mk, &m->Z1, &m->Z2, &m->O, &m->dO, &m->dZ1, &m->dZ2};
    for (float **b : bufs) { cudaFree(*b); *b = nullptr; }
    m->cap = 0;
}

cudaError_t run_forward(pava_mlp *m) {
    forward_kernel<<<m->B, HID>>>(m->P, m->X, m->B, m->Z1, m->Z2, m->O);
    return cudaGetLastError();
}

cudaError_t run_gradient(pava_mlp *m) {
    cudaError_t e = run_forward(m);
    if (e != cudaSuccess) return e;
    backward_kernel<<<m->B, HID>>>(m->P, m->B, m->Z1, m->Z2, m->O, m->T, m->Mk, m->inv_count,
                                   m->dO, m->dZ1, m->dZ2);
    grad_kernel<<<(NP + 255) / 256, 256>>>(m->X, m->B, m->Z1, m->Z2, m->dO, m->dZ1, m->dZ2, m->G);
    loss_kernel<<<1, 256>>>(m->O, m->T, m->Mk, (long long)m->B * OUT, m->inv_count, m->loss);
    return cudaGetLastError();
}

}  // namespace

extern "C" {

pava_status pava_mlp_create(uint64_t seed, pava_mlp **out) {
    if (!out) { set_last_error("out is NULL"); return PAVA_E_INVALID_ARG; }
    *out = nullptr;
    pava_mlp *m = new (std::nothrow) pava_mlp();
    if (!m) return PAVA_E_NOMEM;
    cudaError_t e = cudaMalloc(&m->P, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaMalloc(&m->G, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaMalloc(&m->Mm, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaMalloc(&m->Vv, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaMalloc(&m->mu, sizeof(float) * IN);
    if (e == cudaSuccess) e = cudaMalloc(&m->sd, sizeof(float) * IN);
    if (e == cudaSuccess) e = cudaMalloc(&m->loss, sizeof(float));
    // He-uniform weights (bound sqrt(6 / fan_in)), zero biases, identity normalisation
    std::vector<float> h(NP, 0.f);
    auto fill = [&](int off, int count, int fan_in, uint64_t tag) {
        const float bound = sqrtf(6.f / fan_in);
        for (int q = 0; q < count; ++q) {
            const uint64_t r = mix64(mix64(seed * 0xD6E8FEB86659FD93ull + tag) ^ (uint64_t)q);
            const float u = (float)((double)(r >> 11) * 0x1.0p-53) * 2.f - 1.f;
            h[off + q] = u * bound;
        }
    };
    fill(OW1, HID * IN, IN, 1);
    fill(OW2, HID * HID, HID, 2);
    fill(OW3, OUT * HID, HID, 3);
    std::vector<float> zero(IN, 0.f), one(IN, 1.f);
    if (e == cudaSuccess) e = cudaMemcpy(m->P, h.data(), sizeof(float) * NP, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->Mm, 0, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaMemset(m->Vv, 0, sizeof(float) * NP);
    if (e == cudaSuccess) e = cudaMemcpy(m->mu, zero.data(), sizeof(float) * IN, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->sd, one.data(), sizeof(float) * IN, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        pava_mlp_destroy(m);
        return mfail(e, "mlp create");
    }
    *out = m;
    return PAVA_SUCCESS;
}

pava_status pava_mlp_get_params(const pava_mlp *m, float *params, float *mean12, float *std12) {
    if (!m) { set_last_error("mlp is NULL"); return PAVA_E_INVALID_ARG; }
    cudaError_t e = cudaSuccess;
    if (params) e = cudaMemcpy(params, m->P, sizeof(float) * NP, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && mean12) e = cudaMemcpy(mean12, m->mu, sizeof(float) * IN, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && std12) e = cudaMemcpy(std12, m->sd, sizeof(float) * IN, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? PAVA_SUCCESS : mfail(e, "mlp get");
}

pava_status pava_mlp_set_params(pava_mlp *m, const float *params, const float *mean12,
                                const float *std12) {
    if (!m) { set_last_error("mlp is NULL"); return PAVA_E_INVALID_ARG; }
    if (std12)
        for (int i = 0; i < IN; ++i)
            if (!(std12[i] > 0.f)) { set_last_error("std must be > 0"); return PAVA_E_INVALID_ARG; }
    cudaError_t e = cudaSuccess;
    if (params) {
        e = cudaMemcpy(m->P, params, sizeof(float) * NP, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(m->Mm, 0, sizeof(float) * NP);
        if (e == cudaSuccess) e = cudaMemset(m->Vv, 0, sizeof(float) * NP);
        m->step = 0;
    }
    if (e == cudaSuccess && mean12) e = cudaMemcpy(m->mu, mean12, sizeof(float) * IN, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && std12) e = cudaMemcpy(m->sd, std12, sizeof(float) * IN, cudaMemcpyHostToDevice);
    return e == cudaSuccess ? PAVA_SUCCESS : mfail(e, "mlp set");
}

pava_status pava_mlp_set_batch(pava_mlp *m, int B, const float *X, const float *T,
                               const float *mask) {
    if (!m || !X || B < 1) { set_last_error("mlp, X or B invalid"); return PAVA_E_INVALID_ARG; }
    cudaError_t e = cudaSuccess;
    if (B > m->cap) {
        free_batch(m);
        const size_t b = (size_t)B;
        e = cudaMalloc(&m->X, sizeof(float) * b * IN);
        if (e == cudaSuccess) e = cudaMalloc(&m->T, sizeof(float) * b * OUT);
        if (e == cudaSuccess) e = cudaMalloc(&m->Mk, sizeof(float) * b * OUT);
        if (e == cudaSuccess) e = cudaMalloc(&m->Z1, sizeof(float) * b * HID);
        if (e == cudaSuccess) e = cudaMalloc(&m->Z2, sizeof(float) * b * HID);
        if (e == cudaSuccess) e = cudaMalloc(&m->O, sizeof(float) * b * OUT);
        if (e == cudaSuccess) e = cudaMalloc(&m->dO, sizeof(float) * b * OUT);
        if (e == cudaSuccess) e = cudaMalloc(&m->dZ1, sizeof(float) * b * HID);
        if (e == cudaSuccess) e = cudaMalloc(&m->dZ2, sizeof(float) * b * HID);
        if (e != cudaSuccess) { free_batch(m); return mfail(e, "mlp batch"); }
        m->cap = B;
    }
    m->B = B;
    e = cudaMemcpy(m->X, X, sizeof(float) * (size_t)B * IN, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        normalize_kernel<<<(unsigned)(((long long)B * IN + 255) / 256), 256>>>(m->X, B, m->mu, m->sd);
        e = cudaGetLastError();
    }
    std::vector<float> tt((size_t)B * OUT, 0.f), mk((size_t)B * OUT, 0.f);
    double count = 0;
    if (T) {
        for (size_t q = 0; q < tt.size(); ++q) {
            tt[q] = T[q];
            mk[q] = mask ? mask[q] : 1.f;
            count += mk[q];
        }
    }
    m->inv_count = count > 0 ? (float)(1.0 / count) : 0.f;
    if (e == cudaSuccess) e = cudaMemcpy(m->T, tt.data(), sizeof(float) * tt.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->Mk, mk.data(), sizeof(float) * mk.size(), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? PAVA_SUCCESS : mfail(e, "mlp batch upload");
}

pava_status pava_mlp_forward(pava_mlp *m, float *Y) {
    if (!m || m->B < 1) { set_last_error("no batch set"); return PAVA_E_INVALID_ARG; }
    cudaError_t e = run_forward(m);
    if (e == cudaSuccess && Y)
        e = cudaMemcpy(Y, m->O, sizeof(float) * (size_t)m->B * OUT, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? PAVA_SUCCESS : mfail(e, "mlp forward");
}

pava_status pava_mlp_gradient(pava_mlp *m, float *grad, float *loss) {
    if (!m || m->B < 1) { set_last_error("no batch set"); return PAVA_E_INVALID_ARG; }
    cudaError_t e = run_gradient(m);
    if (e == cudaSuccess && grad) e = cudaMemcpy(grad, m->G, sizeof(float) * NP, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && loss) e = cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? PAVA_SUCCESS : mfail(e, "mlp gradient");
}

pava_status pava_mlp_train(pava_mlp *m, int epochs, float lr, float *loss_hist) {
    if (!m || m->B < 1 || epochs < 0) { set_last_error("no batch set"); return PAVA_E_INVALID_ARG; }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    std::vector<float> hist((size_t)epochs, 0.f);
    cudaError_t e = cudaSuccess;
    for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
        e = run_gradient(m);
        ++m->step;
        const float c1 = 1.f / (1.f - powf(b1, (float)m->step));
        const float c2 = 1.f / (1.f - powf(b2, (float)m->step));
        adam_kernel<<<(NP + 255) / 256, 256>>>(m->P, m->G, m->Mm, m->Vv, lr, b1, b2, eps, c1, c2);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess && loss_hist)
            e = cudaMemcpyAsync(&hist[ep], m->loss, sizeof(float), cudaMemcpyDeviceToHost, nullptr);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess && loss_hist) memcpy(loss_hist, hist.data(), sizeof(float) * hist.size());
    return e == cudaSuccess ? PAVA_SUCCESS : mfail(e, "mlp train");
}

pava_status pava_mlp_destroy(pava_mlp *m) {
    if (!m) return PAVA_SUCCESS;
    free_batch(m);
    cudaFree(m->P); cudaFree(m->G); cudaFree(m->Mm); cudaFree(m->Vv);
    cudaFree(m->mu); cudaFree(m->sd); cudaFree(m->loss);
    delete m;
    return PAVA_SUCCESS;
}

}  // extern "C"
