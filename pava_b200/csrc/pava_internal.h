// Internal declarations shared by the engine's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <string>

#include "../../include/pava_gpu.h"
#include "pava_common.cuh"

namespace pava {

// Per-chunk metadata of the GPU CVR form (128 bytes; one chunk = 32 lanes x S steps).
// The row phase needs only the header; the rest describes the chunk's tail, where the rows
// still open when the chunk ran out of rows are spread evenly over the 32 lanes.
struct CvrMeta {
    ChunkHdr h;
    int i_t;       // first tail step (== S when the chunk has no tail)
    int ntail;     // tail slots (rows still open at i_t, in row order), <= 64
    int n_inprog;  // slots [0, n_inprog) hold rows a lane was working on at i_t
    int next_g;    // slot n_inprog + j holds row r_first + next_g + j
    unsigned cont; // bit k: lane k's first tail element continues lane k-1's last row
    unsigned pad[3];
    unsigned char park[32];        // slot of lane k's row in progress at i_t, 0xff if none
    unsigned char first_slot[32];  // slot of lane k's first tail element
    unsigned pad2[4];
};
static_assert(sizeof(CvrMeta) == 128, "CvrMeta layout");

// Per-slice descriptor of the SELL form (32 rows; 4-step blocks of 128 elements).
struct SellSlice {
    int off;         // first element of the slice in the value and column streams
    int nblk;        // 4-step blocks: the slice's longest row, rounded up to 4, over 4
    int colbase;     // DELTA16: base column of the 16-bit offsets
    unsigned flags;  // bit 0: some row of the slice is padded (padding reads no x); bits 1..31:
                     // the first block holding padding (the shortest row / 4)
};
static_assert(sizeof(SellSlice) == 16, "SellSlice layout");

// Engine handle (behind the opaque pava_handle of the C ABI).
struct Handle {
    int format = 0, precision = 0, index_mode = 0;
    int m = 0, n = 0, nnz = 0, n_empty = 0;
    long long n_aug = 0;     // elements after giving every empty row one zero element
    long long nchunks = 0;   // warp chunks
    long long L = 0;         // elements per chunk (padded space = nchunks * L)
    int S = 0;               // CVR: steps per chunk
    int sigma = 0, G = 0;    // CSR5: elements per lane per tile, tiles per chunk
    long long ntiles = 0;
    int lanes_per_row = 0;   // plain CSR: lanes per row group (GL)
    int col_lanes = 1;       //   lanes across the right-hand sides (KC)
    int cols_per_lane = 1;   //   right-hand sides per lane (KPL)
    int rows_per_tile = 0;   //   rows per warp tile of the persistent launch (TR), or per
                             //   CTA tile with x_window
    int x_window = 0;        //   stage each CTA tile's window of X in shared memory
    int device = 0, sm_count = 0;

    int *arp = nullptr;            // augmented row pointer, m + 2 entries (row m = padding)
    void *vals = nullptr;          // format value stream
    void *cols = nullptr;          // format column stream
    unsigned *flags = nullptr;     // CVR row-end bits / CSR5 row-start descriptors
    void *meta = nullptr;          // per-chunk metadata (CvrMeta or ChunkHdr)
    size_t meta_stride = 0;
    int *tile_ptr = nullptr;       // CSR5 tile -> first row
    int *colbase = nullptr;        // DELTA16: per-chunk base column of the 16-bit offsets
    double *carry_head = nullptr;  // per-chunk partial of a first row shared with the left
    double *carry_tail = nullptr;  // per-chunk partial of a last row shared with the right
    int *rp = nullptr, *ci = nullptr;  // plain CSR form
    void *v = nullptr;                 //   values: double, or float for FP32C

    double convert_ms = 0.0;
    size_t device_bytes = 0;
    int d16_overflow = 0;    // the last conversion found a column outside the 16-bit range
};

// Sets the message pava_last_error() returns on this thread.
void set_last_error(const std::string &msg);

// Device address of the bounds-check error word (three 64-bit words) on the current device in
// builds with PAVA_BOUNDS_CHECK; nullptr in ordinary builds, whose kernels never test it.
unsigned long long *guard_word();

// Device address of the bounded-wait word (two 64-bit words: waits that gave up, and the first
// one's site + 1) on the current device; in every build.  nullptr when it cannot be resolved.
unsigned long long *wait_word();

// CSR5 tiles per chunk.  The persistent grid keeps `warps` warps resident (24 per SM); each
// takes chunks in turn, so a chunk count just above a multiple of `warps` leaves a last wave
// that few warps run.
// Default: 4 tiles per chunk, fewer when that leaves fewer chunks than warps.
inline int csr5_default_tiles(long long tiles, long long warps) {
    return tiles >= 4 * warps ? 4 : (tiles >= 2 * warps ? 2 : 1);
}
// Wave-balanced: the G in 1..8 with the fewest tiles on a warp's critical path,
// ceil(tiles / (G * warps)) * G; the largest G among equals.
inline int csr5_wave_tiles(long long tiles, long long warps) {
    int best = 1;
    long long best_t = -1;
    for (int g = 1; g <= 8; ++g) {
        const long long t = (tiles + g * warps - 1) / (g * warps) * g;
        if (best_t < 0 || t <= best_t) { best_t = t; best = g; }
    }
    return best;
}

// Kernel launchers (stream-ordered; return cudaGetLastError()).
cudaError_t launch_validate(const int *rp, const int *ci, int m, int n, int nnz, int *d_err,
                            cudaStream_t s);
cudaError_t build_augmented_rowptr(const int *rp, int m, long long padded_total, int *arp,
                                   int *d_nempty, cudaStream_t s);

// DELTA16 base column of every warp chunk (h.colbase): the midpoint of the chunk's smallest
// and largest column.
cudaError_t chunk_colbase(const Handle &h, const int *rp, const int *ci, cudaStream_t s);

// Conversions set *ovf (device) to 1 when a 16-bit column offset does not fit.
cudaError_t cvr_convert(Handle &h, const int *rp, const int *ci, const double *v, int *ovf,
                        cudaStream_t s);
cudaError_t cvr_spmv(const Handle &h, const void *x, void *y, cudaStream_t s);

cudaError_t csr5_convert(Handle &h, const int *rp, const int *ci, const double *v, int *ovf,
                         cudaStream_t s);
cudaError_t csr5_spmv(const Handle &h, const void *x, void *y, cudaStream_t s);

cudaError_t carry_fixup(const Handle &h, void *y, cudaStream_t s);

// SELL: sell_plan fills the slice descriptors (h.meta, h.nchunks slices) except their offsets
// and writes the exclusive scan of the slices' block counts to d_blk_off[0..nslices], the total
// to *d_total_blk; sell_fill writes the padded streams and the offsets.
cudaError_t sell_plan(Handle &h, const int *rp, const int *ci, int *d_blk_off, int *d_total_blk,
                      cudaStream_t s);
cudaError_t sell_fill(Handle &h, const int *rp, const int *ci, const double *v,
                      const int *d_blk_off, int *ovf, cudaStream_t s);
cudaError_t sell_spmv(const Handle &h, const void *x, void *y, cudaStream_t s);
// SELL SpMM, Y = A X with X row-major n x k; leading dimensions ldx, ldy in elements.  Lanes per
// row (h.lanes_per_row): 4 (k <= 32), 8 (k <= 64) or 16 (k <= 64); 0 = 4 for k <= 16, else 8.
// sell_spmm_lanes gives the lanes it uses for k, 0 when the handle's choice cannot serve k
// (sell_spmm then returns cudaErrorInvalidValue).
constexpr int SELL_SPMM_MAX_K = 64;
inline int sell_spmm_lanes(int lanes_per_row, int k) {
    const int g = lanes_per_row ? lanes_per_row : (k <= 16 ? 4 : 8);
    if (g == 4) return k <= 32 ? 4 : 0;
    if (g == 8 || g == 16) return k <= SELL_SPMM_MAX_K ? g : 0;
    return 0;
}
cudaError_t sell_spmm(const Handle &h, const void *X, long long ldx, void *Y, long long ldy,
                      int k, cudaStream_t s);

// Plain CSR row-group kernel: y = A x, and Y = A X with X row-major n x k (leading
// dimensions ldx, ldy in elements).
cudaError_t csr_spmv(const Handle &h, const void *x, void *y, cudaStream_t s);
cudaError_t csr_spmm(const Handle &h, const void *X, long long ldx, void *Y, long long ldy,
                     int k, cudaStream_t s);
cudaError_t narrow_to_float(const double *src, float *dst, long long n, cudaStream_t s);

}  // namespace pava
