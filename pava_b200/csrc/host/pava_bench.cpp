// pava_bench: the benchmark loop of pava's main.cpp (conduct_benchmark, main.cpp:554-587) for
// the CVR and CSR5 sections, with the GPU engine in place of the AVX-512 one.
//
//   pava_bench <matrix.mtx> [iterations] [--sell]
//   pava_bench --laplace <grid> [iterations] [--sell]
//   pava_bench --powerlaw <rows> [iterations] [--sell]
//
// --sell adds a third section for the SELL form (no counterpart in main.cpp), or one line
// saying why the form refuses the matrix.
//
// Per section: y is zeroed (initVectors, basicMatrix.cpp:499-520), the engine entry point
// converts, runs the checked SpMV into y and times `iterations` more (printing the
// reference's " Performance <name> CVR|CSR5 <SMs> <convert s> <exec s>" line), then the
// reference's check counts rows off by more than 1 % of y_ref (checkResults,
// basicMatrix.cpp:559-587) against a serial CSR product (referenceSpMV, :538-556).  The CVR
// section keeps main.cpp's guard of both dimensions above 4096 (main.cpp:558).
//
// Beside each Performance line the driver prints one machine-readable record, a JSON object on
// a line of its own starting with {"record": "pava_bench": the section's form and tile
// parameters, convert and exec seconds, GB/s by the compulsory byte model and its fraction of
// the HBM peak (PAVA_HBM_PEAK_GBS, else MEASURED_PEAKS.json two directories above the
// executable, else 6,650 GB/s marked "fallback"), and the error of y against the serial product
// (per-row relative error with the cancellation-aware denominator max(|y_ref|, sum |a x|)).

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "pava_gpu.h"
#include "pava_host.h"

namespace {

int check_results(int m, const double *y, const double *y_ref) {
    int bad = 0;
    for (int r = 0; r < m; ++r) {
        const double d = fabs(y[r] - y_ref[r]);
        if (d > 0.01 * fabs(y_ref[r])) ++bad;
    }
    return bad;
}

void reference_spmv(int m, const int *rp, const int *ci, const double *v, const double *x,
                    double *y, double *absum) {
    for (int r = 0; r < m; ++r) {
        double s = 0.0, a = 0.0;
        for (int j = rp[r]; j < rp[r + 1]; ++j) {
            s += v[j] * x[ci[j]];
            a += fabs(v[j] * x[ci[j]]);
        }
        y[r] = s;
        absum[r] = a;
    }
}

struct Peak {
    double gbs = 6650.0;
    const char *kind = "fallback";
};

// The HBM peak the roofline fraction is taken against.
Peak hbm_peak(const char *argv0) {
    Peak p;
    if (const char *env = getenv("PAVA_HBM_PEAK_GBS")) {
        p.gbs = atof(env);
        p.kind = "env";
        return p;
    }
    std::string dir(argv0);
    const size_t slash = dir.find_last_of('/');
    dir = slash == std::string::npos ? std::string(".") : dir.substr(0, slash);
    FILE *f = fopen((dir + "/../../MEASURED_PEAKS.json").c_str(), "r");
    if (!f) return p;
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
    fclose(f);
    const size_t k = text.find("\"hbm_gbs\"");
    if (k != std::string::npos) {
        const size_t colon = text.find(':', k);
        if (colon != std::string::npos) {
            const double v = atof(text.c_str() + colon + 1);
            if (v > 0) {
                p.gbs = v;
                p.kind = "measured";
            }
        }
    }
    return p;
}

void print_record(const std::string &name, const char *section, const pava_run_record &r, int m,
                  int n, int nnz, const double *y, const double *y_ref, const double *absum,
                  int rows_off, const Peak &peak) {
    double mx = 0.0, mean = 0.0;
    for (int i = 0; i < m; ++i) {
        double den = fabs(y_ref[i]) > absum[i] ? fabs(y_ref[i]) : absum[i];
        if (den < 1e-300) den = 1e-300;
        const double e = fabs(y[i] - y_ref[i]) / den;
        mx = e > mx ? e : mx;
        mean += e;
    }
    mean = m ? mean / m : 0.0;
    const double gbs = r.exec_s > 0 ? r.alg_bytes / r.exec_s / 1e9 : -1.0;
    printf("{\"record\": \"pava_bench\", \"matrix\": \"%s\", \"section\": \"%s\", "
           "\"status\": %d, \"m\": %d, \"n\": %d, \"nnz\": %d, \"format\": %d, "
           "\"precision\": %d, \"index_bytes\": %d, \"steps\": %d, \"sigma\": %d, "
           "\"tiles_per_chunk\": %d, \"chunks\": %lld, \"sms\": %d, \"iterations\": %d, "
           "\"convert_s\": %.6e, \"exec_s\": %.6e, \"alg_bytes\": %.0f, "
           "\"format_bytes\": %.0f, \"GBps\": %.3f, \"peak_GBps\": %.1f, "
           "\"peak_kind\": \"%s\", \"roofline_frac\": %.4f, \"max_rel_err\": %.3e, "
           "\"mean_rel_err\": %.3e, \"rows_off_1pct\": %d}\n",
           name.c_str(), section, r.status, m, n, nnz, r.format, r.precision,
           r.index_mode == PAVA_INDEX_DELTA16 ? 2 : 4, r.steps, r.sigma, r.tiles_per_chunk,
           r.chunks, r.sm_count, r.iterations, r.convert_s, r.exec_s, r.alg_bytes,
           r.format_bytes, gbs, peak.gbs, peak.kind, gbs > 0 ? gbs / peak.gbs : -1.0, mx, mean,
           rows_off);
    fflush(stdout);
}

struct Csr {
    int m = 0, n = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
};

bool load_mtx(const char *path, Csr &A) {
    int m, n, kind, sym;
    long long nz;
    if (pava_mtx_info(path, &m, &n, &nz, &kind, &sym) != 0) return false;
    std::vector<int> rows(nz), cols(nz);
    std::vector<double> vals(nz);
    long long got = 0;
    if (pava_mtx_read(path, rows.data(), cols.data(), vals.data(), &got) != 0) return false;
    A.m = m;
    A.n = n;
    A.rp.assign((size_t)m + 1, 0);
    A.ci.resize(got);
    A.v.resize(got);
    return pava_coo_to_csr(m, n, got, rows.data(), cols.data(), vals.data(), A.rp.data(),
                           A.ci.data(), A.v.data()) == 0;
}

bool generate(const char *kind, int size, Csr &A) {
    if (!strcmp(kind, "--laplace")) {
        A.m = A.n = size * size;
        A.rp.assign((size_t)A.m + 1, 0);
        if (pava_gen_laplace2d_rowptr(size, A.rp.data()) != 0) return false;
        A.ci.resize(A.rp[A.m]);
        A.v.resize(A.rp[A.m]);
        return pava_gen_laplace2d_fill(size, A.rp.data(), A.ci.data(), A.v.data()) == 0;
    }
    if (!strcmp(kind, "--powerlaw")) {
        A.m = A.n = size;
        A.rp.assign((size_t)A.m + 1, 0);
        if (pava_gen_powerlaw_rowptr(A.m, A.n, 16.0, 1.5, 200000, 0.02, 1, A.rp.data()) != 0)
            return false;
        A.ci.resize(A.rp[A.m]);
        A.v.resize(A.rp[A.m]);
        return pava_gen_powerlaw_fill(A.m, A.n, 1, A.rp.data(), A.ci.data(), A.v.data()) == 0;
    }
    return false;
}

}  // namespace

int main(int argc, char **argv) {
    bool with_sell = false;  // a trailing --sell asks for the SELL section
    if (argc >= 2 && !strcmp(argv[argc - 1], "--sell")) {
        with_sell = true;
        --argc;
    }
    if (argc < 2) {
        fprintf(stderr, "usage: %s <matrix.mtx> [iterations] | --laplace <grid> [it] | "
                        "--powerlaw <rows> [it], then optionally --sell\n", argv[0]);
        return 2;
    }
    Csr A;
    std::string name;
    int arg = 2;
    if (argv[1][0] == '-' && argv[1][1] == '-') {
        if (argc < 3 || !generate(argv[1], atoi(argv[2]), A)) {
            fprintf(stderr, "cannot generate %s\n", argv[1]);
            return 2;
        }
        name = std::string(argv[1] + 2) + "_" + argv[2];
        arg = 3;
    } else {
        if (!load_mtx(argv[1], A)) {
            fprintf(stderr, "cannot read %s\n", argv[1]);
            return 2;
        }
        name = argv[1];
        const size_t slash = name.find_last_of('/');
        if (slash != std::string::npos) name = name.substr(slash + 1);
    }
    const int iters = argc > arg ? atoi(argv[arg]) : 1000;  // LARGE_ITERS, main.cpp:55
    if (pava_init(0) != PAVA_SUCCESS) {
        fprintf(stderr, "no usable GPU: %s\n", pava_last_error());
        return 1;
    }
    const int nnz = A.rp[A.m];
    std::vector<double> x(A.n), y(A.m), y_ref(A.m), absum(A.m);
    pava_init_vectors(A.m, A.n, x.data(), y.data(), y_ref.data());
    reference_spmv(A.m, A.rp.data(), A.ci.data(), A.v.data(), x.data(), y_ref.data(),
                   absum.data());
    const Peak peak = hbm_peak(argv[0]);
    const pava_csr csr{A.m, A.n, nnz, A.rp.data(), A.ci.data(), A.v.data(), 0};
    pava_opts opts;
    memset(&opts, 0, sizeof(opts));
    opts.index_mode = PAVA_INDEX_AUTO;  // what conduct_cvr_gpu / conduct_csr5_gpu use
    printf("matrix %s: %d x %d, %d nonzeros\n", name.c_str(), A.m, A.n, nnz);
    std::vector<char> cname(name.begin(), name.end());
    cname.push_back('\0');

    int failures = 0;
    printf("**************\n      CVR      \n**************\n");
    if (A.m > 4096 && A.n > 4096) {
        pava_init_vectors(A.m, A.n, nullptr, y.data(), nullptr);
        pava_run_record rec;
        const int st = pava_conduct(PAVA_FORMAT_CVR, &csr, x.data(), y.data(), cname.data(),
                                    iters, &opts, &rec);
        const int bad = check_results(A.m, y.data(), y_ref.data());
        printf("CVR status %d, rows off by more than 1%%: %d\n", st, bad);
        print_record(name, "CVR", rec, A.m, A.n, nnz, y.data(), y_ref.data(), absum.data(), bad,
                     peak);
        failures += (st != 0) + (bad != 0);
    } else {
        printf(" Performance %s %s %d %f %f \n", cname.data(), "CVR", 0, -1.0, -1.0);
    }
    printf("**************\n     CSR5     \n**************\n");
    pava_init_vectors(A.m, A.n, nullptr, y.data(), nullptr);
    pava_run_record rec;
    const int st = pava_conduct(PAVA_FORMAT_CSR5, &csr, x.data(), y.data(), cname.data(), iters,
                                &opts, &rec);
    const int bad = check_results(A.m, y.data(), y_ref.data());
    printf("CSR5 status %d, rows off by more than 1%%: %d\n", st, bad);
    print_record(name, "CSR5", rec, A.m, A.n, nnz, y.data(), y_ref.data(), absum.data(), bad,
                 peak);
    failures += (st != 0) + (bad != 0);
    if (with_sell) {
        printf("**************\n     SELL     \n**************\n");
        pava_init_vectors(A.m, A.n, nullptr, y.data(), nullptr);
        pava_run_record srec;
        const int sst = pava_conduct(PAVA_FORMAT_SELL, &csr, x.data(), y.data(), cname.data(),
                                     iters, &opts, &srec);
        if (sst == PAVA_E_UNSUPPORTED_PARAMS) {  // the slices would pad too much: not a failure
            printf("SELL refuses the matrix: %s\n", pava_last_error());
        } else {
            const int sbad = check_results(A.m, y.data(), y_ref.data());
            printf("SELL status %d, rows off by more than 1%%: %d\n", sst, sbad);
            print_record(name, "SELL", srec, A.m, A.n, nnz, y.data(), y_ref.data(),
                         absum.data(), sbad, peak);
            failures += (sst != 0) + (sbad != 0);
        }
    }
    return failures ? 1 : 0;
}
