// GPU CSR5: CSR -> CSR5 conversion and CSR5 SpMV for sm_100a.
//
// The reference's CSR5 (csr5/, anonymouslib for AVX-512) cuts the nnz range into tiles of
// omega lanes x sigma elements (omega = 8 there), stores a tile pointer (the tile's first row,
// format_avx512.h:8-28), per-lane bit flags marking row starts (format_avx512.h:85-121) and
// transposes each tile so that step i of all lanes is contiguous (format_avx512.h:365-426).
// The SpMV does a per-lane segmented sum, a cross-lane scan (hscan_avx512) and adds the
// partial row that crosses thread boundaries through a calibrator (csr5_spmv_avx512.h:52-308).
//
// Here omega is the warp (32 lanes) and sigma is a multiple of 4 (default 16):
//  * a tile descriptor is one 32-bit row-start mask per lane.  The y_offset and
//    scansum_offset fields the reference packs beside the flags (format_avx512.h:123-233) are
//    recomputed per tile from the masks with a warp scan and ballot, which costs a few
//    instructions instead of descriptor bytes.
//  * empty rows are given one zero element in column -1 (see k_cvr.cu), so every row of a
//    tile is consecutive and no descriptor-offset table (format_avx512.h:271-363) is needed.
//  * a warp walks G consecutive tiles (a chunk) carrying the open row in registers; the
//    chunk's shared first/last rows go to the carry slots combined by k_fixup.cu, the
//    deterministic form of the calibrator (csr5_spmv_avx512.h:292-308).  The reference's
//    serial tail partition (:311-342) does not exist: the last tile is padded.
//
// Tile t (32*sigma elements, element (lane l, step i) = original position t*32*sigma +
// l*sigma + i):
//   values  at t*32*sigma + (i/VP)*32*VP + VP*l + i%VP
//   columns at t*32*sigma + (i/CP)*32*CP + CP*l + i%CP
//   desc[t*32 + l]  bit i: element (l, i) is the first element of a row
//   tile_ptr[t]     row of element (0, 0)

#include "pava_internal.h"

namespace pava {

namespace {

template <int VP, int CP, typename VT>
__global__ void __launch_bounds__(256)
csr5_convert_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                    const double *__restrict__ v, const int *__restrict__ arp, int m,
                    long long ntiles, int sigma, VT *__restrict__ vals, int *__restrict__ cols,
                    unsigned *__restrict__ desc, int *__restrict__ tile_ptr) {
    const int lane = threadIdx.x & 31;
    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= ntiles) return;
    const long long tbase = t * 32LL * sigma;
    const long long e0 = tbase + (long long)lane * sigma;
    const int nr = m + 2;
    int row = upper_bound_m1(arp, nr, e0);
    if (lane == 0) tile_ptr[t] = row;
    int rbase = 0;
    bool dummy = true;
    auto src_of = [&](int r) {
        if (r >= m) { dummy = true; rbase = 0; return; }
        const int a = rp[r];
        dummy = (rp[r + 1] == a);
        rbase = a - arp[r];
    };
    src_of(row);
    int next_start = arp[row + 1];
    unsigned F = 0;
    for (int i = 0; i < sigma; ++i) {
        const long long e = e0 + i;
        while ((long long)next_start <= e) {
            ++row;
            src_of(row);
            next_start = arp[row + 1];
        }
        if ((long long)arp[row] == e) F |= 1u << i;
        double val = 0.0;
        int col = -1;
        if (!dummy) {
            val = v[e + rbase];
            col = ci[e + rbase];
        }
        vals[tbase + (i / VP) * 32 * VP + VP * lane + (i % VP)] = (VT)val;
        cols[tbase + (i / CP) * 32 * CP + CP * lane + (i % CP)] = col;
    }
    desc[t * 32 + lane] = F;
}

__global__ void chunk_hdr_kernel(const int *__restrict__ arp, int m, long long nchunks,
                                 long long L, ChunkHdr *__restrict__ hdr) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    const long long s = c * L, e = s + L;
    const int r_first = upper_bound_m1(arp, m + 2, s);
    const int r_last = upper_bound_m1(arp, m + 2, e - 1);
    unsigned sh = 0;
    if ((long long)arp[r_first] < s) sh |= 1u;
    if ((long long)arp[r_last + 1] > e) sh |= 2u;
    hdr[c].r_first = r_first;
    hdr[c].nrows = r_last - r_first + 1;
    hdr[c].shared = sh;
    hdr[c].aux = 0;
}

constexpr int SPMV_WARPS = 8;

// CSR5 SpMV, FP64: one warp per chunk of G tiles of 32 x SIGMA elements.
template <int SIGMA>
__global__ void __launch_bounds__(SPMV_WARPS * 32)
csr5_spmv_f64_kernel(const ChunkHdr *__restrict__ hdr, const int *__restrict__ tile_ptr,
                     const unsigned *__restrict__ desc, const double *__restrict__ vals,
                     const int *__restrict__ cols, const double *__restrict__ x,
                     double *__restrict__ y, double *__restrict__ carry_head,
                     double *__restrict__ carry_tail, long long nchunks, int G, int m) {
    constexpr int TE = 32 * SIGMA;  // elements per tile
    constexpr int NQ = SIGMA / 4;   // 4-step groups per tile
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
    const long long nwarps = (long long)gridDim.x * SPMV_WARPS;

    for (long long c = (long long)blockIdx.x * SPMV_WARPS + w; c < nchunks; c += nwarps) {
        const ChunkHdr H = hdr[c];
        const int r_first = H.r_first, r_last = H.r_first + H.nrows - 1;
        const unsigned shared = H.shared;
        int carry_row = (shared & 1u) ? r_first : -1;
        double carry_val = 0.0;
        for (int tt = 0; tt < G; ++tt) {
            const long long t = c * G + tt;
            const int row_start = tile_ptr[t];
            const unsigned F = ld_stream(desc + t * 32 + lane, pf);
            const double2 *vb = reinterpret_cast<const double2 *>(vals + t * TE);
            const int4 *cb = reinterpret_cast<const int4 *>(cols + t * TE);
            const int b00 = (int)(__shfl_sync(FULL, F, 0) & 1u);
            const int nst = __popc(F);
            const int excl = warp_excl_scan(nst, lane);
            const int total = __shfl_sync(FULL, excl + nst, 31);
            int rowcur = row_start + excl - b00;  // row open when the lane starts
            double acc = 0.0, hpiece = 0.0;
            bool seen = false;
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const int4 cc = ld_stream(cb + q * 32 + lane, pf);
                const double2 va = ld_stream(vb + (2 * q) * 32 + lane, pf);
                const double2 vc = ld_stream(vb + (2 * q + 1) * 32 + lane, pf);
                const double xx[4] = {gather_x(x, cc.x, pl), gather_x(x, cc.y, pl),
                                      gather_x(x, cc.z, pl), gather_x(x, cc.w, pl)};
                const double vv[4] = {va.x, va.y, vc.x, vc.y};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int i = q * 4 + k;
                    if ((F >> i) & 1u) {
                        if (seen) {
                            if (rowcur < m) y[rowcur] = acc;
                        } else {
                            hpiece = acc;
                            seen = true;
                        }
                        ++rowcur;
                        acc = 0.0;
                    }
                    acc = fma(vv[k], xx[k], acc);
                }
            }
            if (!seen) hpiece = acc;
            const double tl = seen ? acc : 0.0;
            const unsigned sm = __ballot_sync(FULL, seen);
            const double Hs = seg_suffix(hpiece, !seen, lane);
            double Hn = __shfl_down_sync(FULL, Hs, 1);
            if (lane == 31) Hn = 0.0;
            const double H0 = __shfl_sync(FULL, Hs, 0);
            if (sm == 0) {
                carry_val += H0;  // the whole tile continues the open row
            } else {
                const int lstar = 31 - __clz(sm);
                const double own_l = tl + Hn;
                if (seen && lane != lstar && rowcur < m) y[rowcur] = own_l;
                const double own = __shfl_sync(FULL, own_l, lstar);
                if (carry_row >= 0 && lane == 0)
                    flush_row(carry_row, carry_val + H0, r_first, r_last, shared, c, y,
                              carry_head, carry_tail, m);
                carry_row = row_start + total - b00;
                carry_val = own;
            }
        }
        if (carry_row >= 0 && lane == 0)
            flush_row(carry_row, carry_val, r_first, r_last, shared, c, y, carry_head,
                      carry_tail, m);
    }
}

}  // namespace

cudaError_t csr5_convert(Handle &h, const int *rp, const int *ci, const double *v,
                         cudaStream_t s) {
    if (h.ntiles <= 0) return cudaSuccess;
    const long long blocks = (h.ntiles * 32 + 255) / 256;
    if (h.precision != PAVA_PREC_FP64) return cudaErrorInvalidValue;
    csr5_convert_kernel<2, 4, double><<<(unsigned)blocks, 256, 0, s>>>(
        rp, ci, v, h.arp, h.m, h.ntiles, h.sigma, (double *)h.vals, (int *)h.cols, h.flags,
        h.tile_ptr);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    chunk_hdr_kernel<<<(unsigned)((h.nchunks + 255) / 256), 256, 0, s>>>(
        h.arp, h.m, h.nchunks, h.L, (ChunkHdr *)h.meta);
    return cudaGetLastError();
}

cudaError_t csr5_spmv(const Handle &h, const void *x, void *y, cudaStream_t s) {
    if (h.nchunks <= 0) return cudaSuccess;
    if (h.precision != PAVA_PREC_FP64) return cudaErrorInvalidValue;
    const long long want = (h.nchunks + SPMV_WARPS - 1) / SPMV_WARPS;
    const long long cap = (long long)h.sm_count * 8;
    const unsigned grid = (unsigned)(want < cap ? want : cap);
#define PAVA_CSR5_LAUNCH(SG)                                                                \
    csr5_spmv_f64_kernel<SG><<<grid, SPMV_WARPS * 32, 0, s>>>(                              \
        (const ChunkHdr *)h.meta, h.tile_ptr, h.flags, (const double *)h.vals,              \
        (const int *)h.cols, (const double *)x, (double *)y, h.carry_head, h.carry_tail,    \
        h.nchunks, h.G, h.m)
    switch (h.sigma) {
        case 8: PAVA_CSR5_LAUNCH(8); break;
        case 12: PAVA_CSR5_LAUNCH(12); break;
        case 16: PAVA_CSR5_LAUNCH(16); break;
        case 24: PAVA_CSR5_LAUNCH(24); break;
        case 32: PAVA_CSR5_LAUNCH(32); break;
        default: return cudaErrorInvalidValue;
    }
#undef PAVA_CSR5_LAUNCH
    return cudaGetLastError();
}

}  // namespace pava
