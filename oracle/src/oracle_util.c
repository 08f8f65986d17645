/*
 * ORACLE -- test infrastructure only (never linked by the product).
 * Long-double CSR reference, the cancellation-aware per-row error metric and the reference's
 * 1 % check (utils/basicMatrix.cpp:538-587).
 */
#include <math.h>
#include "oracle.h"

void oracle_csr_ref(int m, const int *rp, const int *ci, const double *v, const double *x,
                    double *y_ref, double *absum) {
#pragma omp parallel for schedule(dynamic, 1024)
    for (int i = 0; i < m; i++) {
        long double s = 0.0L, a = 0.0L;
        for (int j = rp[i]; j < rp[i + 1]; j++) {
            long double p = (long double)v[j] * (long double)x[ci[j]];
            s += p;
            a += fabsl(p);
        }
        y_ref[i] = (double)s;
        if (absum) absum[i] = (double)a;
    }
}

long long oracle_rel_error(int m, const double *y, const double *y_ref, const double *absum,
                           double tol, double *max_rel, double *mean_rel) {
    double mx = 0.0, sum = 0.0;
    long long bad = 0;
    for (int i = 0; i < m; i++) {
        double d = fabs(y[i] - y_ref[i]);
        double den = fabs(y_ref[i]);
        if (absum && absum[i] > den) den = absum[i];
        double r = den > 0.0 ? d / den : d;
        if (!(r <= tol)) bad++; /* NaN counts as bad */
        if (r > mx || r != r) mx = r;
        sum += r;
    }
    if (max_rel) *max_rel = mx;
    if (mean_rel) *mean_rel = m > 0 ? sum / m : 0.0;
    return bad;
}

long long oracle_check_results(int m, const double *y, const double *y_ref) {
    long long err = 0;
    for (int i = 0; i < m; i++)
        if (fabs(y_ref[i] - y[i]) > 0.01 * fabs(y_ref[i])) err++;
    return err;
}
