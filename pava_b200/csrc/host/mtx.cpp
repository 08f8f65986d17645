// Matrix Market coordinate I/O and COO -> CSR (include/pava_host.h).

#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "pava_host.h"

namespace {

struct MtxHeader {
    int m = 0, n = 0;
    long long stored = 0;
    int kind = 0;       // 0 real, 1 integer, 2 pattern, 3 complex
    int symmetric = 0;  // symmetric, skew-symmetric or hermitian: mirror off-diagonal entries
    int skew = 0;
};

int read_header(FILE *f, MtxHeader *h) {
    char line[4096];
    if (!fgets(line, sizeof line, f)) return -3;
    char banner[64], object[64], format[64], field[64], sym[64];
    if (sscanf(line, "%63s %63s %63s %63s %63s", banner, object, format, field, sym) != 5) return -3;
    if (strcasecmp(banner, "%%MatrixMarket") != 0) return -3;
    if (strcasecmp(object, "matrix") != 0 || strcasecmp(format, "coordinate") != 0) return -3;
    if (!strcasecmp(field, "real")) h->kind = 0;
    else if (!strcasecmp(field, "integer")) h->kind = 1;
    else if (!strcasecmp(field, "pattern")) h->kind = 2;
    else if (!strcasecmp(field, "complex")) h->kind = 3;
    else return -3;
    if (!strcasecmp(sym, "general")) h->symmetric = 0;
    else if (!strcasecmp(sym, "symmetric") || !strcasecmp(sym, "hermitian")) h->symmetric = 1;
    else if (!strcasecmp(sym, "skew-symmetric")) { h->symmetric = 1; h->skew = 1; }
    else return -3;
    do {
        if (!fgets(line, sizeof line, f)) return -3;
    } while (line[0] == '%' || line[strspn(line, " \t\r\n")] == '\0');
    long long m, n, nz;
    if (sscanf(line, "%lld %lld %lld", &m, &n, &nz) != 3 || m < 0 || n < 0 || nz < 0) return -3;
    if (m > 2147483647LL || n > 2147483647LL) return -15;
    h->m = (int)m;
    h->n = (int)n;
    h->stored = nz;
    return 0;
}

}  // namespace

extern "C" {

int pava_mtx_info(const char *path, int *m, int *n, long long *nnz_alloc, int *kind,
                  int *symmetric) {
    FILE *f = fopen(path, "r");
    if (!f) return -10;
    MtxHeader h;
    int rc = read_header(f, &h);
    fclose(f);
    if (rc) return rc;
    if (m) *m = h.m;
    if (n) *n = h.n;
    if (nnz_alloc) *nnz_alloc = h.symmetric ? 2 * h.stored : h.stored;
    if (kind) *kind = h.kind;
    if (symmetric) *symmetric = h.symmetric;
    return 0;
}

int pava_mtx_read(const char *path, int *rows, int *cols, double *vals, long long *nnz) {
    FILE *f = fopen(path, "r");
    if (!f) return -10;
    MtxHeader h;
    int rc = read_header(f, &h);
    if (rc) { fclose(f); return rc; }
    long long k = 0;
    char line[4096];
    for (long long e = 0; e < h.stored; ++e) {
        if (!fgets(line, sizeof line, f)) { fclose(f); return -3; }
        if (line[0] == '%') { --e; continue; }
        long long r, c;
        double a = 1.0, b = 0.0;
        int got;
        if (h.kind == 2) got = sscanf(line, "%lld %lld", &r, &c) == 2;
        else if (h.kind == 3) got = sscanf(line, "%lld %lld %lf %lf", &r, &c, &a, &b) >= 3;
        else got = sscanf(line, "%lld %lld %lf", &r, &c, &a) == 3;
        if (!got || r < 1 || c < 1 || r > h.m || c > h.n) { fclose(f); return -11; }
        rows[k] = (int)(r - 1);  // 1-based file, 0-based COO
        cols[k] = (int)(c - 1);
        vals[k] = a;
        ++k;
        if (h.symmetric && r != c) {
            rows[k] = (int)(c - 1);
            cols[k] = (int)(r - 1);
            vals[k] = h.skew ? -a : a;
            ++k;
        }
    }
    fclose(f);
    if (nnz) *nnz = k;
    return 0;
}

int pava_mtx_write(const char *path, int m, int n, const int *rp, const int *ci,
                   const double *v) {
    FILE *f = fopen(path, "w");
    if (!f) return -10;
    fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n");
    fprintf(f, "%d %d %d\n", m, n, rp[m]);
    for (int r = 0; r < m; ++r)
        for (int j = rp[r]; j < rp[r + 1]; ++j) fprintf(f, "%d %d %.17g\n", r + 1, ci[j] + 1, v[j]);
    int rc = ferror(f) ? -10 : 0;
    fclose(f);
    return rc;
}

int pava_coo_to_csr(int m, int n, long long nnz, const int *rows, const int *cols,
                    const double *vals, int *rp, int *ci, double *v) {
    if (m < 0 || n < 0 || nnz < 0 || nnz > 2147483647LL) return -10;
    std::vector<long long> cnt((size_t)m + 1, 0);
    for (long long k = 0; k < nnz; ++k) {
        if (rows[k] < 0 || rows[k] >= m || cols[k] < 0 || cols[k] >= n) return -11;
        ++cnt[(size_t)rows[k] + 1];
    }
    for (int r = 0; r < m; ++r) cnt[(size_t)r + 1] += cnt[r];
    for (int r = 0; r <= m; ++r) rp[r] = (int)cnt[r];
    std::vector<long long> pos(cnt.begin(), cnt.end() - 1);
    std::vector<long long> perm((size_t)nnz);
    for (long long k = 0; k < nnz; ++k) perm[(size_t)pos[(size_t)rows[k]]++] = k;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int r = 0; r < m; ++r) {
        auto b = perm.begin() + rp[r], e = perm.begin() + rp[r + 1];
        std::stable_sort(b, e, [&](long long a, long long c) { return cols[a] < cols[c]; });
        for (int j = rp[r]; j < rp[r + 1]; ++j) {
            ci[j] = cols[perm[(size_t)j]];
            v[j] = vals[perm[(size_t)j]];
        }
    }
    return 0;
}

}  // extern "C"
