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
//    chunk's shared first/last rows go to the carry slots combined by k_support.cu, the
//    deterministic form of the calibrator (csr5_spmv_avx512.h:292-308).  The reference's
//    serial tail partition (:311-342) does not exist: the last tile is padded.
//
// Tile t (32*sigma elements; element (lane l, step i) = original position t*32*sigma +
// l*sigma + i) holds its values and columns in the 4-step block layout of k_stream.cuh, so a
// chunk of G tiles is one run of G*sigma/4 blocks;
//   desc[t*32 + l]  bit i: element (l, i) is the first element of a row
//   tile_ptr[t]     row of element (0, 0)

#include "k_stream.cuh"
#include "pava_internal.h"

namespace pava {

namespace {

template <typename IT> __device__ __forceinline__ IT enc_col(int col, int base, int *ovf);
template <> __device__ __forceinline__ int enc_col<int>(int col, int, int *) { return col; }
template <> __device__ __forceinline__ short enc_col<short>(int col, int base, int *ovf) {
    if (col < 0) return DELTA_NONE;
    const int d = col - base;
    if (d < -32767 || d > 32767) { atomicOr(ovf, 1); return DELTA_NONE; }
    return (short)d;
}

template <typename VT, typename IT>
__global__ void __launch_bounds__(256)
csr5_convert_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                    const double *__restrict__ v, const int *__restrict__ arp, int m,
                    long long ntiles, int sigma, int G, VT *__restrict__ vals,
                    IT *__restrict__ cols, unsigned *__restrict__ desc,
                    int *__restrict__ tile_ptr, ChunkHdr *__restrict__ hdr,
                    const int *__restrict__ colbase, int *ovf) {
    const int lane = threadIdx.x & 31;
    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= ntiles) return;
    const int nr = m + 2;
    const long long tbase = t * 32LL * sigma;
    const int col_base = sizeof(IT) == 2 ? colbase[t / G] : 0;  // of the 16-bit offsets
    const long long e0 = tbase + (long long)lane * sigma;
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
    bool reads_none = false;  // some element of the lane reads no x
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
        } else {
            reads_none = true;
        }
        vals[tbase + vals_offset<VT>(i, lane)] = (VT)val;
        cols[tbase + cols_offset(i, lane)] = enc_col<IT>(col, col_base, ovf);
    }
    desc[t * 32 + lane] = F;
    if (reads_none) atomicOr(&hdr[t / G].aux, 1);
}

// Chunk headers.  aux bits 1..31: the base column of the chunk's 16-bit offsets (colbase,
// when the form has them), read with the header; bit 0 (set by csr5_convert_kernel, which
// runs after this kernel): the chunk holds elements that read no x (the zero element of an
// empty row, or the padding of the last chunk); chunks without them skip that check.
__global__ void chunk_hdr_kernel(const int *__restrict__ arp, const int *__restrict__ colbase,
                                 int m, long long nchunks, long long L,
                                 ChunkHdr *__restrict__ hdr) {
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
    hdr[c].aux = colbase ? (int)((unsigned)colbase[c] << 1) : 0;
}

// Tile end: the cross-lane combine of the lanes' open row pieces.  head is the piece a lane
// adds to the row open at its start (its whole sum when no row starts in the lane), tail the
// sum since the lane's last row start (seen: a row starts in the lane), rowcur the row of that
// tail, next_row the row open at the tile's end.  Rows that end in the tile go to y (or to
// the chunk's carry slots); the open row's sum stays in carry_row / carry_val.  The FP64
// kernel has the same steps inline: calling this helper there changed its register allocation
// and doubled its spills at 80 registers.
__device__ __forceinline__ void tile_combine(double head, double tail, bool seen, int rowcur,
                                             int next_row, int lane, int r_first, int r_last,
                                             unsigned shared, long long c, double *y,
                                             double *carry_head, double *carry_tail, int m,
                                             int &carry_row, double &carry_val,
                                             unsigned long long *err) {
    const unsigned sm = __ballot_sync(FULL, seen);
    const double Hs = seg_suffix(head, !seen, lane);
    double Hn = __shfl_down_sync(FULL, Hs, 1);
    if (lane == 31) Hn = 0.0;
    const double H0 = __shfl_sync(FULL, Hs, 0);
    if (sm == 0) {
        carry_val += H0;  // the whole tile continues the open row
    } else {
        const int lstar = 31 - __clz(sm);
        const double own_l = tail + Hn;
        if (seen && lane != lstar && rowcur < m && guard(err, rowcur >= 0, G_Y, rowcur))
            y[rowcur] = own_l;
        const double own = __shfl_sync(FULL, own_l, lstar);
        if (carry_row >= 0 && lane == 0)
            flush_row(carry_row, carry_val + H0, r_first, r_last, shared, c, y, carry_head,
                      carry_tail, m, err);
        carry_row = next_row;
        carry_val = own;
    }
}

#ifndef PAVA_CSR5_MINB32
#define PAVA_CSR5_MINB32 3
#endif
#ifndef PAVA_CSR5_MINB
#define PAVA_CSR5_MINB 3
#endif
constexpr int SPMV_WARPS = 8;

// CSR5 SpMV (FP64 values; the FP32 form is csr5_spmv_f32_kernel below): one warp per chunk of
// G tiles, walked as one pipelined run of 4-step blocks
// (values two blocks ahead, columns three, x one); tile descriptors one tile ahead.
//
// Row ends inside a tile: when no lane of the warp starts more than KSTK rows in the tile
// (the usual case), an element that starts a row parks the lane's finished piece in the
// lane's next shared-memory slot (a predicated store) and restarts the accumulator (a select),
// so the step has no branch; at the tile end piece 0 (the end of the row the lane started
// with) joins the cross-lane combine and pieces 1 .. k-1, rows that start and end in the
// lane, go to y.  Other tiles write each finished row as it ends.
template <int SIGMA, typename VT, typename IT>
__global__ void __launch_bounds__(SPMV_WARPS * 32, sizeof(VT) == 8 ? PAVA_CSR5_MINB : PAVA_CSR5_MINB32)
csr5_spmv_kernel(const ChunkHdr *__restrict__ hdr, const int *__restrict__ tile_ptr,
                 const unsigned *__restrict__ desc, const VT *__restrict__ vals,
                 const IT *__restrict__ cols, const VT *__restrict__ x,
                 double *__restrict__ y, double *__restrict__ carry_head,
                 double *__restrict__ carry_tail, long long nchunks, int G, int m, int n,
                 unsigned long long *err) {
    constexpr int NBT = SIGMA / 4;  // blocks per tile
    // the carry fixup that follows may launch now; it waits for this grid to finish
    asm volatile("griddepcontrol.launch_dependents;");
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
    const long long nwarps = (long long)gridDim.x * SPMV_WARPS;
    (void)w;
    constexpr int KSTK = 4;
    constexpr unsigned SLOT = SPMV_WARPS * 32 * 8;  // bytes between a thread's slots
    __shared__ __align__(16) double s_piece[KSTK * SPMV_WARPS * 32];
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(&s_piece[threadIdx.x]);

    for (long long c = (long long)blockIdx.x * SPMV_WARPS + w; c < nchunks; c += nwarps) {
        const ChunkHdr H = hdr[c];
        const int r_first = H.r_first, r_last = H.r_first + H.nrows - 1;
        const unsigned shared = H.shared;
        int carry_row = (shared & 1u) ? r_first : -1;
        double carry_val = 0.0;
        const long long t0 = c * G;
        const VT *vb = vals + t0 * 32 * SIGMA;
        const IT *cb = cols + t0 * 32 * SIGMA;
        const int xbase = sizeof(IT) == 2 ? (int)((unsigned)H.aux >> 1) : 0;  // offsets' base
        const VT *xb = x + xbase;
        const int xlo = -xbase, xhi = n - xbase;  // the offsets that stay inside x
        const int NB = G * NBT;

        CBlk<IT> c1 = CBlk<IT>::load(cb, 1, lane, pf);
        CBlk<IT> c2 = CBlk<IT>::load(cb, NB > 2 ? 2 : 1, lane, pf);
        VBlk<VT> v0 = VBlk<VT>::load(vb, 0, lane, pf), v1 = VBlk<VT>::load(vb, 1, lane, pf);
        VT x0[4];
        {
            const CBlk<IT> c0 = CBlk<IT>::load(cb, 0, lane, pf);
#pragma unroll
            for (int q = 0; q < 4; ++q) x0[q] = c0.gather(q, xb, pl, xlo, xhi, err);
        }
        unsigned Fn = ld_stream(desc + t0 * 32 + lane, pf);
        int rsn = tile_ptr[t0];

        unsigned F = 0;
        int rs = 0, b00 = 0, total = 0, rowcur = 0;
        Acc<VT> acc;
        double hpiece = 0.0;
        bool seen = false;
        int tt = 0;
        bool fast = false;
        int nst = 0, row0 = 0;
        unsigned sp = sbase;
#pragma unroll 1
        for (int blk = 0; blk < NB; ++blk) {
            CBlk<IT> cn = c2;
            VBlk<VT> vn = v1;
            if (blk + 3 < NB) cn = CBlk<IT>::load(cb, blk + 3, lane, pf);
            if (blk + 2 < NB) vn = VBlk<VT>::load(vb, blk + 2, lane, pf);
            VT x1[4];
            if (blk + 1 < NB) {
#pragma unroll
                for (int q = 0; q < 4; ++q) x1[q] = c1.gather(q, xb, pl, xlo, xhi, err);
            }
            const int qb = blk % NBT;
            if (qb == 0) {  // tile start
                F = Fn;
                rs = rsn;
                if (tt + 1 < G) {
                    Fn = ld_stream(desc + (t0 + tt + 1) * 32 + lane, pf);
                    rsn = tile_ptr[t0 + tt + 1];
                }
                b00 = (int)(__shfl_sync(FULL, F, 0) & 1u);
                nst = __popc(F);
                const int excl = warp_excl_scan(nst, lane);
                total = __shfl_sync(FULL, excl + nst, 31);
                rowcur = rs + excl - b00;  // row open when the lane starts
                row0 = rowcur;
                acc.reset();
                hpiece = 0.0;
                seen = false;
                fast = !__any_sync(FULL, nst > KSTK);
                sp = sbase;
            }
            const unsigned Fb = F >> (qb * 4);
            if (fast) {  // row ends park the piece in the lane's shared slots: no branch
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const bool st = (Fb >> q) & 1u;
                    acc.push(sp, st);
                    sp += st ? SLOT : 0u;
                    acc.add_restart(v0.get(q), x0[q], st);
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if ((Fb >> q) & 1u) {
                        if (seen) {
                            if (rowcur < m && guard(err, rowcur >= 0, G_Y, rowcur)) y[rowcur] = acc.value();
                        } else {
                            hpiece = acc.value();
                            seen = true;
                        }
                        ++rowcur;
                        acc.reset();
                    }
                    acc.add(v0.get(q), x0[q]);
                }
            }
            if (qb == NBT - 1) {  // tile end: combine the lanes' open pieces
                if (fast) {
                    seen = nst > 0;
                    if (seen) hpiece = Acc<VT>::piece_at(sbase);
                    for (int k2 = 1; k2 < nst; ++k2)
                        if (row0 + k2 < m && guard(err, row0 + k2 >= 0 && k2 < KSTK, G_Y, row0 + k2))
                        y[row0 + k2] = Acc<VT>::piece_at(sbase + k2 * SLOT);
                    rowcur = row0 + nst;
                }
                if (!seen) hpiece = acc.value();
                const double tl = seen ? acc.value() : 0.0;
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
                    if (seen && lane != lstar && rowcur < m && guard(err, rowcur >= 0, G_Y, rowcur))
            y[rowcur] = own_l;
                    const double own = __shfl_sync(FULL, own_l, lstar);
                    if (carry_row >= 0 && lane == 0)
                        flush_row(carry_row, carry_val + H0, r_first, r_last, shared, c, y,
                                  carry_head, carry_tail, m, err);
                    carry_row = rs + total - b00;
                    carry_val = own;
                }
                ++tt;
            }
            c1 = c2; c2 = cn;
            v0 = v1; v1 = vn;
#pragma unroll
            for (int q = 0; q < 4; ++q) x0[q] = x1[q];
        }
        if (carry_row >= 0 && lane == 0)
            flush_row(carry_row, carry_val, r_first, r_last, shared, c, y, carry_head,
                      carry_tail, m, err);
    }
}

template <bool B> struct Flag { static constexpr bool value = B; };

// CSR5 SpMV, FP32-compensated form: the same walk with a tile's sigma/4 blocks unrolled, so
// the block pipeline rotates by register renaming instead of moves, and the fast / slow
// choice and the tile-boundary checks are made once per tile instead of once per block.  The
// compensated add makes this form instruction-issue bound, where the saved instructions are
// time; the FP64 form is bandwidth bound, and unrolled it spills, so it keeps the block loop.
template <int SIGMA, typename IT>
__global__ void __launch_bounds__(SPMV_WARPS * 32, PAVA_CSR5_MINB32)
csr5_spmv_f32_kernel(const ChunkHdr *__restrict__ hdr, const int *__restrict__ tile_ptr,
                     const unsigned *__restrict__ desc, const float *__restrict__ vals,
                     const IT *__restrict__ cols, const float *__restrict__ x,
                     double *__restrict__ y, double *__restrict__ carry_head,
                     double *__restrict__ carry_tail, long long nchunks, int G, int m, int n,
                     unsigned long long *err) {
    using VT = float;
    constexpr int NBT = SIGMA / 4;  // blocks per tile
    // the carry fixup that follows may launch now; it waits for this grid to finish
    asm volatile("griddepcontrol.launch_dependents;");
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
    const long long nwarps = (long long)gridDim.x * SPMV_WARPS;
    constexpr int KSTK = 4;
    constexpr unsigned SLOT = SPMV_WARPS * 32 * 8;  // bytes between a thread's slots
    __shared__ __align__(16) double s_piece[KSTK * SPMV_WARPS * 32];
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(&s_piece[threadIdx.x]);

    for (long long c = (long long)blockIdx.x * SPMV_WARPS + w; c < nchunks; c += nwarps) {
        const ChunkHdr H = hdr[c];
        const int r_first = H.r_first, r_last = H.r_first + H.nrows - 1;
        const unsigned shared = H.shared;
        // chunks without elements that read no x skip the gather's test (16-bit offsets and
        // tiles of 24 or 32 steps; the other forms gained nothing from it or spilled)
        constexpr bool SKIP = sizeof(IT) == 2 && SIGMA >= 24;
        const bool chk = !SKIP || (H.aux & 1);
        int carry_row = (shared & 1u) ? r_first : -1;
        double carry_val = 0.0;
        const long long t0 = c * G;
        const VT *vb = vals + t0 * 32 * SIGMA;
        const IT *cb = cols + t0 * 32 * SIGMA;
        const int xbase = sizeof(IT) == 2 ? (int)((unsigned)H.aux >> 1) : 0;  // offsets' base
        const VT *xb = x + xbase;
        const int xlo = -xbase, xhi = n - xbase;  // the offsets that stay inside x
        const int NB = G * NBT;

        CBlk<IT> c1 = CBlk<IT>::load(cb, 1, lane, pf);
        CBlk<IT> c2 = CBlk<IT>::load(cb, NB > 2 ? 2 : 1, lane, pf);
        VBlk<VT> v0 = VBlk<VT>::load(vb, 0, lane, pf), v1 = VBlk<VT>::load(vb, 1, lane, pf);
        VT x0[4];
        {
            const CBlk<IT> c0 = CBlk<IT>::load(cb, 0, lane, pf);
#pragma unroll
            for (int q = 0; q < 4; ++q) x0[q] = c0.gather(q, xb, pl, xlo, xhi, err);
        }
        unsigned Fn = ld_stream(desc + t0 * 32 + lane, pf);
        int rsn = tile_ptr[t0];

#pragma unroll 1
        for (int tt = 0; tt < G; ++tt) {
            // tile start: the lanes' row-start masks give each lane its first row
            const unsigned F = Fn;
            const int rs = rsn;
            if (tt + 1 < G) {
                Fn = ld_stream(desc + (t0 + tt + 1) * 32 + lane, pf);
                rsn = tile_ptr[t0 + tt + 1];
            }
            const int b00 = (int)(__shfl_sync(FULL, F, 0) & 1u);
            const int nst = __popc(F);
            const int excl = warp_excl_scan(nst, lane);
            const int total = __shfl_sync(FULL, excl + nst, 31);
            const int row0 = rs + excl - b00;  // row open when the lane starts
            const int rem = G - 1 - tt;        // tiles after this one
            int rowcur = row0;
            Acc<VT> acc;
            double hpiece = 0.0;
            bool seen = false;

            // The tile's blocks.  Block qb prefetches block qb + d of the chunk (columns d = 3,
            // values 2, x 1); that block lies (qb + d) / NBT tiles ahead, so only prefetches
            // past this tile compare against the tiles left.  CHK: the chunk has elements that
            // read no x, so each gather tests its column.
            auto walk = [&](auto fast_tag, auto chk_tag) {
                constexpr bool FAST = decltype(fast_tag)::value;
                constexpr bool CHK = decltype(chk_tag)::value;
                unsigned sp = sbase;
#pragma unroll
                for (int qb = 0; qb < NBT; ++qb) {
                    CBlk<IT> cn = c2;
                    VBlk<VT> vn = v1;
                    if ((qb + 3) / NBT == 0 || rem >= (qb + 3) / NBT)
                        cn = CBlk<IT>::load(cb, tt * NBT + qb + 3, lane, pf);
                    if ((qb + 2) / NBT == 0 || rem >= (qb + 2) / NBT)
                        vn = VBlk<VT>::load(vb, tt * NBT + qb + 2, lane, pf);
                    VT x1[4];
                    if ((qb + 1) / NBT == 0 || rem >= (qb + 1) / NBT) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            x1[q] = CHK ? c1.gather(q, xb, pl, xlo, xhi, err)
                                        : c1.gather_all(q, xb, pl, xlo, xhi, err);
                    }
                    if (FAST) {  // row ends park the piece in the lane's shared slots
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const bool st = (F >> (qb * 4 + q)) & 1u;
                            acc.push(sp, st);
                            sp += st ? SLOT : 0u;
                            acc.add_restart(v0.get(q), x0[q], st);
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            if ((F >> (qb * 4 + q)) & 1u) {
                                if (seen) {
                                    if (rowcur < m && guard(err, rowcur >= 0, G_Y, rowcur)) y[rowcur] = acc.value();
                                } else {
                                    hpiece = acc.value();
                                    seen = true;
                                }
                                ++rowcur;
                                acc.reset();
                            }
                            acc.add(v0.get(q), x0[q]);
                        }
                    }
                    c1 = c2; c2 = cn;
                    v0 = v1; v1 = vn;
#pragma unroll
                    for (int q = 0; q < 4; ++q) x0[q] = x1[q];
                }
            };
            if (!__any_sync(FULL, nst > KSTK)) {
                if (!SKIP || chk) walk(Flag<true>{}, Flag<true>{});
                else walk(Flag<true>{}, Flag<false>{});
                seen = nst > 0;
                if (seen) hpiece = Acc<VT>::piece_at(sbase);
                for (int k2 = 1; k2 < nst; ++k2)
                    if (row0 + k2 < m && guard(err, row0 + k2 >= 0 && k2 < KSTK, G_Y, row0 + k2))
                        y[row0 + k2] = Acc<VT>::piece_at(sbase + k2 * SLOT);
                rowcur = row0 + nst;
            } else {
                walk(Flag<false>{}, Flag<true>{});
            }
            const double a = acc.value();
            tile_combine(seen ? hpiece : a, seen ? a : 0.0, seen, rowcur, rs + total - b00,
                         lane, r_first, r_last, shared, c, y, carry_head, carry_tail, m,
                         carry_row, carry_val, err);
        }
        if (carry_row >= 0 && lane == 0)
            flush_row(carry_row, carry_val, r_first, r_last, shared, c, y, carry_head,
                      carry_tail, m, err);
    }
}

template <typename VT, typename IT>
cudaError_t convert_t(Handle &h, const int *rp, const int *ci, const double *v, int *ovf,
                      cudaStream_t s) {
    chunk_hdr_kernel<<<(unsigned)((h.nchunks + 255) / 256), 256, 0, s>>>(
        h.arp, h.colbase, h.m, h.nchunks, h.L, (ChunkHdr *)h.meta);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    const long long blocks = (h.ntiles * 32 + 255) / 256;
    csr5_convert_kernel<VT, IT><<<(unsigned)blocks, 256, 0, s>>>(
        rp, ci, v, h.arp, h.m, h.ntiles, h.sigma, h.G, (VT *)h.vals, (IT *)h.cols, h.flags,
        h.tile_ptr, (ChunkHdr *)h.meta, h.colbase, ovf);
    return cudaGetLastError();
}

template <int SG, typename VT, typename IT>
void launch_sg(const Handle &h, unsigned grid, const void *x, void *y, cudaStream_t s) {
    if constexpr (sizeof(VT) == 4)
        csr5_spmv_f32_kernel<SG, IT><<<grid, SPMV_WARPS * 32, 0, s>>>(
            (const ChunkHdr *)h.meta, h.tile_ptr, h.flags, (const float *)h.vals,
            (const IT *)h.cols, (const float *)x, (double *)y, h.carry_head,
            h.carry_tail, h.nchunks, h.G, h.m, h.n, guard_word());
    else
        csr5_spmv_kernel<SG, VT, IT><<<grid, SPMV_WARPS * 32, 0, s>>>(
            (const ChunkHdr *)h.meta, h.tile_ptr, h.flags, (const VT *)h.vals,
            (const IT *)h.cols, (const VT *)x, (double *)y, h.carry_head,
            h.carry_tail, h.nchunks, h.G, h.m, h.n, guard_word());
}

template <typename VT, typename IT>
cudaError_t spmv_t(const Handle &h, const void *x, void *y, cudaStream_t s) {
    const long long want = (h.nchunks + SPMV_WARPS - 1) / SPMV_WARPS;
    const long long cap = (long long)h.sm_count * (sizeof(VT) == 8 ? PAVA_CSR5_MINB : PAVA_CSR5_MINB32);
    const unsigned grid = (unsigned)(want < cap ? want : cap);
    switch (h.sigma) {
        case 8: launch_sg<8, VT, IT>(h, grid, x, y, s); break;
        case 12: launch_sg<12, VT, IT>(h, grid, x, y, s); break;
        case 16: launch_sg<16, VT, IT>(h, grid, x, y, s); break;
        case 24: launch_sg<24, VT, IT>(h, grid, x, y, s); break;
        case 32: launch_sg<32, VT, IT>(h, grid, x, y, s); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t csr5_convert(Handle &h, const int *rp, const int *ci, const double *v, int *ovf,
                         cudaStream_t s) {
    if (h.ntiles <= 0) return cudaSuccess;
    const bool f32 = h.precision == PAVA_PREC_FP32C, d16 = h.index_mode == PAVA_INDEX_DELTA16;
    if (!f32 && !d16) return convert_t<double, int>(h, rp, ci, v, ovf, s);
    if (!f32 && d16) return convert_t<double, short>(h, rp, ci, v, ovf, s);
    if (f32 && !d16) return convert_t<float, int>(h, rp, ci, v, ovf, s);
    return convert_t<float, short>(h, rp, ci, v, ovf, s);
}

cudaError_t csr5_spmv(const Handle &h, const void *x, void *y, cudaStream_t s) {
    if (h.nchunks <= 0) return cudaSuccess;
    const bool f32 = h.precision == PAVA_PREC_FP32C, d16 = h.index_mode == PAVA_INDEX_DELTA16;
    if (!f32 && !d16) return spmv_t<double, int>(h, x, y, s);
    if (!f32 && d16) return spmv_t<double, short>(h, x, y, s);
    if (f32 && !d16) return spmv_t<float, int>(h, x, y, s);
    return spmv_t<float, short>(h, x, y, s);
}

}  // namespace pava
