// Seeded synthetic matrix generators (include/pava_host.h).  Deterministic for any thread
// count: every random number is a hash of (seed, stream, counter).

#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "pava_host.h"

namespace {

inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Counter-based draw: stream = row (or a tagged row), ctr = element counter.
inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t ctr) {
    return splitmix64(splitmix64(seed * 0xD6E8FEB86659FD93ull + stream) ^ (ctr * 0x9E3779B97F4A7C15ull));
}
inline double unif(uint64_t seed, uint64_t stream, uint64_t ctr) {  // [0, 1)
    return (double)(draw(seed, stream, ctr) >> 11) * 0x1.0p-53;
}
inline double normal(uint64_t seed, uint64_t stream, uint64_t ctr) {  // Box-Muller
    const double u1 = 1.0 - unif(seed, stream, 2 * ctr);  // (0, 1]
    const double u2 = unif(seed, stream, 2 * ctr + 1);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

constexpr uint64_t TAG_LEN = 1ull << 40;   // stream tags keep lengths, columns, values apart
constexpr uint64_t TAG_COL = 2ull << 40;
constexpr uint64_t TAG_VAL = 3ull << 40;

int finish_rowptr(int m, const std::vector<long long> &len, int *rp) {
    long long acc = 0;
    rp[0] = 0;
    for (int r = 0; r < m; ++r) {
        acc += len[r];
        if (acc > 2147483000LL) return -15;  // PAVA_E_TOO_LARGE
        rp[r + 1] = (int)acc;
    }
    return 0;
}

// L distinct columns in [0, n), sorted, for row r.
void distinct_sorted(int L, int n, uint64_t seed, uint64_t stream, int *out) {
    if (L <= 0) return;
    if ((long long)L * 2 > n) {  // selection sampling over all n columns (Knuth, Algorithm S)
        int need = L, k = 0;
        for (int c = 0; c < n && need > 0; ++c) {
            const double u = unif(seed, stream, (uint64_t)c);
            if ((double)(n - c) * u < (double)need) {
                out[k++] = c;
                --need;
            }
        }
        return;
    }
    std::vector<int> buf;
    buf.reserve((size_t)L + 16);
    uint64_t ctr = 0;
    while ((int)buf.size() < L) {
        const int want = L - (int)buf.size();
        for (int i = 0; i < want; ++i)
            buf.push_back((int)(draw(seed, stream, ctr++) % (uint64_t)n));
        std::sort(buf.begin(), buf.end());
        buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
    }
    memcpy(out, buf.data(), sizeof(int) * (size_t)L);
}

}  // namespace

extern "C" {

int pava_gen_laplace2d_rowptr(int g, int *rp) {
    if (g <= 0 || (long long)g * g > 400000000LL) return -10;
    const int m = g * g;
    rp[0] = 0;
    long long acc = 0;
    for (int r = 0; r < m; ++r) {
        const int i = r / g, j = r % g;
        acc += 1 + (i > 0) + (i < g - 1) + (j > 0) + (j < g - 1);
        rp[r + 1] = (int)acc;
    }
    return 0;
}

int pava_gen_laplace2d_fill(int g, const int *rp, int *ci, double *v) {
    const int m = g * g;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < m; ++r) {
        const int i = r / g, j = r % g;
        int k = rp[r];
        if (i > 0) { ci[k] = r - g; v[k++] = -1.0; }
        if (j > 0) { ci[k] = r - 1; v[k++] = -1.0; }
        ci[k] = r; v[k++] = 4.0;
        if (j < g - 1) { ci[k] = r + 1; v[k++] = -1.0; }
        if (i < g - 1) { ci[k] = r + g; v[k++] = -1.0; }
    }
    return 0;
}

int pava_gen_powerlaw_rowptr(int m, int n, double mean, double sigma, int cap, double p_empty,
                             uint64_t seed, int *rp) {
    if (m < 0 || n <= 0 || cap < 1) return -10;
    std::vector<long long> len((size_t)m);
    const double mu = log(mean) - 0.5 * sigma * sigma;
    const int lim = cap < n ? cap : n;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < m; ++r) {
        if (unif(seed, TAG_LEN + (uint64_t)r, 0) < p_empty) { len[r] = 0; continue; }
        double l = exp(mu + sigma * normal(seed, TAG_LEN + (uint64_t)r, 1));
        long long L = llround(l);
        if (L < 1) L = 1;
        if (L > lim) L = lim;
        len[r] = L;
    }
    return finish_rowptr(m, len, rp);
}

int pava_gen_powerlaw_fill(int m, int n, uint64_t seed, const int *rp, int *ci, double *v) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int r = 0; r < m; ++r) {
        const int a = rp[r], L = rp[r + 1] - a;
        distinct_sorted(L, n, seed, TAG_COL + (uint64_t)r, ci + a);
        for (int k = 0; k < L; ++k) v[a + k] = normal(seed, TAG_VAL + (uint64_t)r, (uint64_t)k);
    }
    return 0;
}

int pava_gen_stencil27_rowptr(int g, int *rp) {
    if (g <= 0 || (long long)g * g * g > 200000000LL) return -10;
    const long long m = (long long)g * g * g;
    rp[0] = 0;
    long long acc = 0;
    for (long long r = 0; r < m; ++r) {
        const int i = (int)(r / ((long long)g * g)), j = (int)((r / g) % g), k = (int)(r % g);
        const int ni = 1 + (i > 0) + (i < g - 1), nj = 1 + (j > 0) + (j < g - 1),
                  nk = 1 + (k > 0) + (k < g - 1);
        acc += ni * nj * nk;
        if (acc > 2147483000LL) return -15;
        rp[r + 1] = (int)acc;
    }
    return 0;
}

int pava_gen_stencil27_fill(int g, uint64_t seed, const int *rp, int *ci, double *v) {
    const long long m = (long long)g * g * g;
    const long long gg = (long long)g * g;
#pragma omp parallel for schedule(static)
    for (long long r = 0; r < m; ++r) {
        const int i = (int)(r / gg), j = (int)((r / g) % g), k = (int)(r % g);
        int p = rp[r];
        int diag = -1;
        double absum = 0.0;
        uint64_t ctr = 0;
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
                for (int dk = -1; dk <= 1; ++dk) {
                    const int ii = i + di, jj = j + dj, kk = k + dk;
                    if (ii < 0 || ii >= g || jj < 0 || jj >= g || kk < 0 || kk >= g) continue;
                    ci[p] = (int)(ii * gg + (long long)jj * g + kk);
                    if (di == 0 && dj == 0 && dk == 0) {
                        diag = p;
                        v[p] = 0.0;
                    } else {
                        const float off = (float)(-unif(seed, TAG_VAL + (uint64_t)r, ctr++));
                        v[p] = (double)off;
                        absum += fabs((double)off);
                    }
                    ++p;
                }
        v[diag] = (double)(float)(1.01 * absum);
    }
    return 0;
}

int pava_gen_banded_rowptr(int m, int h, int per_row, int *rp) {
    if (m < 0 || h < 0 || per_row < 0) return -10;
    rp[0] = 0;
    long long acc = 0;
    for (int r = 0; r < m; ++r) {
        const int lo = r - h < 0 ? 0 : r - h, hi = r + h >= m ? m - 1 : r + h;
        const int W = hi - lo + 1;
        acc += per_row < W ? per_row : W;
        if (acc > 2147483000LL) return -15;
        rp[r + 1] = (int)acc;
    }
    return 0;
}

int pava_gen_banded_fill(int m, int h, uint64_t seed, const int *rp, int *ci, double *v) {
#pragma omp parallel for schedule(static)
    for (int r = 0; r < m; ++r) {
        const int lo = r - h < 0 ? 0 : r - h, hi = r + h >= m ? m - 1 : r + h;
        const int W = hi - lo + 1, a = rp[r], L = rp[r + 1] - a;
        std::vector<int> band((size_t)W);
        for (int t = 0; t < W; ++t) band[t] = lo + t;
        for (int t = 0; t < L; ++t) {  // partial Fisher-Yates
            const int pick = t + (int)(draw(seed, TAG_COL + (uint64_t)r, (uint64_t)t) % (uint64_t)(W - t));
            std::swap(band[t], band[pick]);
        }
        std::sort(band.begin(), band.begin() + L);
        for (int t = 0; t < L; ++t) {
            ci[a + t] = band[t];
            v[a + t] = normal(seed, TAG_VAL + (uint64_t)r, (uint64_t)t);
        }
    }
    return 0;
}

int pava_gen_random_rowptr(int m, int n, double mean, uint64_t seed, int *rp) {
    if (m < 0 || n <= 0) return -10;
    std::vector<long long> len((size_t)m);
    const double lim = exp(-mean);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < m; ++r) {  // Poisson by multiplying uniforms (Knuth)
        long long k = 0;
        double p = 1.0;
        uint64_t ctr = 0;
        do {
            ++k;
            p *= unif(seed, TAG_LEN + (uint64_t)r, ctr++);
        } while (p > lim && k < 100000);
        long long L = k - 1;
        if (L > n) L = n;
        len[r] = L;
    }
    return finish_rowptr(m, len, rp);
}

int pava_gen_random_fill(int m, int n, uint64_t seed, const int *rp, int *ci, double *v) {
    return pava_gen_powerlaw_fill(m, n, seed, rp, ci, v);
}

int pava_gen_blockdiag_rowptr(int m, int bmin, int bmax, uint64_t seed, int *rp) {
    if (m < 0 || bmin < 1 || bmax < bmin) return -10;
    rp[0] = 0;
    long long acc = 0;
    int r = 0;
    uint64_t blk = 0;
    while (r < m) {
        int b = bmin + (int)(draw(seed, TAG_LEN, blk++) % (uint64_t)(bmax - bmin + 1));
        if (b > m - r) b = m - r;
        for (int t = 0; t < b; ++t) {
            acc += b;
            if (acc > 2147483000LL) return -15;
            rp[r + t + 1] = (int)acc;
        }
        r += b;
    }
    return 0;
}

int pava_gen_blockdiag_fill(int m, uint64_t seed, const int *rp, int *ci, double *v) {
    // A row of block [b0, b0+B) has length B and starts at b0 * B + (r - b0) * B; find b0 by
    // walking back while lengths stay equal is O(B); instead rebuild block starts serially.
    std::vector<int> start((size_t)m);
    int r = 0;
    while (r < m) {
        const int B = rp[r + 1] - rp[r];
        for (int t = 0; t < B && r + t < m; ++t) start[r + t] = r;
        r += B > 0 ? B : 1;
    }
#pragma omp parallel for schedule(static)
    for (int q = 0; q < m; ++q) {
        const int a = rp[q], L = rp[q + 1] - a, b0 = start[q];
        for (int t = 0; t < L; ++t) {
            ci[a + t] = b0 + t;
            v[a + t] = normal(seed, TAG_VAL + (uint64_t)q, (uint64_t)t);
        }
    }
    return 0;
}

int pava_gen_uniform(int n, double lo, double hi, uint64_t seed, int fp32, double *x) {
    if (n < 0) return -10;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double t = lo + (hi - lo) * unif(seed, 0, (uint64_t)i);
        x[i] = fp32 ? (double)(float)t : t;
    }
    return 0;
}

void pava_init_vectors(int m, int n, double *x, double *y, double *y_ref) {
    if (y) for (int i = 0; i < m; ++i) y[i] = 0.0;
    if (y_ref) for (int i = 0; i < m; ++i) y_ref[i] = 0.0;
    if (x) for (int i = 0; i < n; ++i) x[i] = (double)(i % 3);
}

}  // extern "C"
