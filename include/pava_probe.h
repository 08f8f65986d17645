/*
 * pava_probe.h -- measurement aids of the pava B200 SpMV engine (libpava_probe.so).
 *
 * No counterpart in the reference: these kernels compute nothing a user needs.  They measure
 * the two costs of an SpMV on a matrix with scattered columns apart from each other -- reading
 * the value and column streams, and gathering x -- so that the SpMV kernels' times can be set
 * against max(stream floor, gather floor) on the same matrix.
 */
#ifndef PAVA_PROBE_H
#define PAVA_PROBE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One launch of a floor kernel over nnz elements in CSR order (device arrays; vals and cols
 * 16-byte aligned, every column in [0, n)), blocks_per_sm x SMs blocks of `threads` threads:
 *   mode 0  streams: reads vals (8 B) and cols (4 B) per element, no x
 *   mode 1  gathers: one x[hash(i, seed) mod n] per element, no streams
 *   mode 2  reads cols and gathers x[cols[i]]
 *   mode 3  reads vals and cols and gathers x[cols[i]] (a dot product without rows)
 * `out` receives one double per warp (pava_probe_floor_out_len entries).  Returns 0, -10 for
 * an invalid argument or -12 for a CUDA error. */
int pava_probe_floor(int mode, const double *vals, const int *cols, const double *x,
                     long long nnz, int n, unsigned long long seed, int blocks_per_sm,
                     int threads, double *out, void *stream);
long long pava_probe_floor_out_len(int blocks_per_sm, int threads);

/* The gathers of mode 1 (x[hash(i, seed) mod n], the first nnz rounded down to 32 elements)
 * fetched by the TMA engine: x (16-byte aligned, n even) viewed as n / 2 rows of 16 bytes under
 * a 2-D tensor map, cp.async.bulk.tensor tile::gather4 into shared memory, bounded mbarrier
 * waits (a wait that gives up counts in *wait_fail, device memory).  blocks_per_sm x SMs blocks
 * of 256 threads; `out` receives one double per warp (pava_probe_floor_out_len(blocks_per_sm,
 * 256) entries), summing to mode 1's total over the same elements.  Returns 0, -10 or -12. */
int pava_probe_gather_tma(const double *x, long long nnz, int n, unsigned long long seed,
                          int blocks_per_sm, double *out, unsigned long long *wait_fail,
                          void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PAVA_PROBE_H */
