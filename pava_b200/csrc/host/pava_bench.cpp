// pava_bench: the benchmark loop of pava's main.cpp (conduct_benchmark, main.cpp:554-587) for
// the CVR and CSR5 sections, with the GPU engine in place of the AVX-512 one.
//
//   pava_bench <matrix.mtx> [iterations]
//   pava_bench --laplace <grid> [iterations]
//   pava_bench --powerlaw <rows> [iterations]
//
// Per section: y is zeroed (initVectors, basicMatrix.cpp:499-520), the engine entry point
// converts, runs the checked SpMV into y and times `iterations` more (printing the
// reference's " Performance <name> CVR|CSR5 <SMs> <convert s> <exec s>" line), then the
// reference's check counts rows off by more than 1 % of y_ref (checkResults,
// basicMatrix.cpp:559-587) against a serial CSR product (referenceSpMV, :538-556).  The CVR
// section keeps main.cpp's guard of both dimensions above 4096 (main.cpp:558).

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
                    double *y) {
    for (int r = 0; r < m; ++r) {
        double s = 0.0;
        for (int j = rp[r]; j < rp[r + 1]; ++j) s += v[j] * x[ci[j]];
        y[r] = s;
    }
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
    if (argc < 2) {
        fprintf(stderr, "usage: %s <matrix.mtx> [iterations] | --laplace <grid> [it] | "
                        "--powerlaw <rows> [it]\n", argv[0]);
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
    std::vector<double> x(A.n), y(A.m), y_ref(A.m);
    pava_init_vectors(A.m, A.n, x.data(), y.data(), y_ref.data());
    reference_spmv(A.m, A.rp.data(), A.ci.data(), A.v.data(), x.data(), y_ref.data());
    printf("matrix %s: %d x %d, %d nonzeros\n", name.c_str(), A.m, A.n, nnz);
    std::vector<char> cname(name.begin(), name.end());
    cname.push_back('\0');

    int failures = 0;
    printf("**************\n      CVR      \n**************\n");
    if (A.m > 4096 && A.n > 4096) {
        pava_init_vectors(A.m, A.n, nullptr, y.data(), nullptr);
        const int st = conduct_cvr_gpu(A.m, A.n, nnz, A.rp.data(), A.ci.data(), A.v.data(),
                                       x.data(), y.data(), 1, cname.data(), iters);
        const int bad = check_results(A.m, y.data(), y_ref.data());
        printf("CVR status %d, rows off by more than 1%%: %d\n", st, bad);
        failures += (st != 0) + (bad != 0);
    } else {
        printf(" Performance %s %s %d %f %f \n", cname.data(), "CVR", 0, -1.0, -1.0);
    }
    printf("**************\n     CSR5     \n**************\n");
    pava_init_vectors(A.m, A.n, nullptr, y.data(), nullptr);
    const int st = conduct_csr5_gpu(A.m, A.n, nnz, A.rp.data(), A.ci.data(), A.v.data(),
                                    x.data(), y.data(), 1.0, cname.data(), iters);
    const int bad = check_results(A.m, y.data(), y_ref.data());
    printf("CSR5 status %d, rows off by more than 1%%: %d\n", st, bad);
    failures += (st != 0) + (bad != 0);
    return failures ? 1 : 0;
}
