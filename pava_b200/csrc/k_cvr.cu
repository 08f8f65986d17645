// GPU CVR: CSR -> CVR conversion and CVR SpMV for sm_100a.
//
// The reference's CVR (cvr/cvr.h) vectorises over 8 AVX-512 lanes: each lane takes the next
// row when its current one ends (pre_processing, cvr/cvr.h:756-905), records where rows end
// (cvr/cvr.h:857-872), and once rows run out lets idle lanes steal work (cvr/cvr.h:906-989).
// Here the lanes are the 32 lanes of a warp and the unit of work is a chunk of 32 x S
// elements of the nnz range (nnz-balanced, like the per-thread split of cvr/cvr.h:602-645):
//
//  * row phase: lane k starts on row r_first + k; whenever lanes finish, they take the next
//    rows in lane order, so a lane's row is r_first + g with g tracked by ballot/popc.  One bit
//    per element marks the element that ends the lane's current row (the GPU form of the
//    reference's (position, row) records): the SpMV stores the lane's accumulator into y
//    there.  Rows a lane finishes are summed in CSR order, one FMA per element.
//  * tail: when a lane finishes and no row is left to take, the rest of the chunk -- the open
//    rows' remaining elements, in row order -- is spread evenly over the 32 lanes (the GPU
//    form of the reference's stealing).  Partial sums meet in shared memory through a
//    fixed-order segmented suffix scan, so the result does not depend on timing.
//  * a chunk's first / last row may continue in the neighbouring chunk; their partial sums go
//    to per-chunk carry slots that k_support.cu adds in chunk order (the reference adds them
//    with `omp atomic`, cvr/cvr.h:1415,1717,1855).
//
// Empty rows are given one element of value 0 in column -1 (which reads no x), so that every
// row is visited and written: y = A x overwrites all of y on every call.  The last chunk is
// padded with such elements, which belong to a padding row m whose sum is dropped.
//
// Streams of chunk c (L = 32*S elements; the 4-step block layout of k_stream.cuh):
//   values  at c*L + vals_offset(i, k), columns at c*L + cols_offset(i, k)
//   flags   word w of lane k at c*S + 32*w + k, bit i%32 of word i/32

#include "k_stream.cuh"
#include "pava_internal.h"

namespace pava {

namespace {

// Source of augmented element e of `row` in the caller's CSR.
struct RowSrc {
    int base;    // rp[row] - arp[row]
    bool dummy;  // empty row or padding row: (0, -1)
};

__device__ __forceinline__ RowSrc row_src(const int *rp, const int *arp, int m, int row) {
    RowSrc r;
    if (row >= m) { r.base = 0; r.dummy = true; return r; }
    const int a = rp[row];
    r.dummy = (rp[row + 1] == a);
    r.base = a - arp[row];
    return r;
}

template <typename IT> __device__ __forceinline__ IT encode_col(int col, int base, int *ovf);
template <> __device__ __forceinline__ int encode_col<int>(int col, int, int *) { return col; }
template <> __device__ __forceinline__ short encode_col<short>(int col, int base, int *ovf) {
    if (col < 0) return DELTA_NONE;
    const int d = col - base;
    if (d < -32767 || d > 32767) { atomicOr(ovf, 1); return DELTA_NONE; }
    return (short)d;
}

template <typename VT, typename IT>
__device__ __forceinline__ void put_elem(VT *vals, IT *cols, long long cbase, int i, int lane,
                                         const int *ci, const double *v, int e, RowSrc src,
                                         int col_base, int *ovf) {
    double val = 0.0;
    int col = -1;
    if (!src.dummy) {
        val = v[e + src.base];
        col = ci[e + src.base];
    }
    vals[cbase + vals_offset<VT>(i, lane)] = (VT)val;
    cols[cbase + cols_offset(i, lane)] = encode_col<IT>(col, col_base, ovf);
}

constexpr int CONV_WARPS = 4;

template <typename VT, typename IT>
__global__ void __launch_bounds__(CONV_WARPS * 32)
cvr_convert_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                   const double *__restrict__ v, const int *__restrict__ arp, int m,
                   long long nchunks, int S, VT *__restrict__ vals, IT *__restrict__ cols,
                   unsigned *__restrict__ flags, CvrMeta *__restrict__ meta,
                   const int *__restrict__ colbase, int *ovf) {
    __shared__ int s_len[CONV_WARPS][64];
    __shared__ int s_src[CONV_WARPS][64];
    __shared__ int s_row[CONV_WARPS][64];
    __shared__ int s_off[CONV_WARPS][65];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long c = (long long)blockIdx.x * CONV_WARPS + w;
    if (c >= nchunks) return;  // warp-uniform
    const long long L = 32LL * S;
    const long long s = c * L, e = s + L;
    const int nr = m + 2;  // arp entries (rows 0..m, m = padding row)
    const int r_first = upper_bound_m1(arp, nr, s);
    const int r_last = upper_bound_m1(arp, nr, e - 1);
    const int nrows = r_last - r_first + 1;
    const int col_base = sizeof(IT) == 2 ? colbase[c] : 0;  // of the 16-bit offsets
    const unsigned lt = lanemask_lt();

    int g = lane, row = -1, cur = 0, rem = 0;
    RowSrc src{0, true};
    auto take = [&](int r) {
        const int a = arp[r], b = arp[r + 1];
        cur = (int)((long long)a > s ? a : s);
        rem = (int)(((long long)b < e ? b : e) - cur);
        src = row_src(rp, arp, m, r);
    };
    if (lane < nrows) { row = r_first + lane; take(row); }
    int next_g = nrows < 32 ? nrows : 32;
    int i_t = S;
    unsigned fword = 0;
    unsigned *fb = flags + c * S;
    int i = 0;
    for (; i < S; ++i) {
        const bool need = (rem == 0);
        const unsigned b = __ballot_sync(FULL, need);
        if (b) {
            if (__popc(b) > nrows - next_g) { i_t = i; break; }
            if (need) {
                g = next_g + __popc(b & lt);
                row = r_first + g;
                take(row);
            }
            next_g += __popc(b);
        }
        put_elem<VT, IT>(vals, cols, s, i, lane, ci, v, cur, src, col_base, ovf);
        ++cur;
        --rem;
        if (rem == 0) fword |= 1u << (i & 31);
        if ((i & 31) == 31) { fb[(i >> 5) * 32 + lane] = fword; fword = 0; }
    }

    int ntail = 0, n_in = 0, park = 0xff, first_slot = 0;
    unsigned contm = 0;
    if (i_t < S) {
        const int T = S - i_t;
        const bool inprog = rem > 0;
        const unsigned ip = __ballot_sync(FULL, inprog);
        n_in = __popc(ip);
        int rank = 0;
        for (int j = 0; j < 32; ++j) {
            const int gj = __shfl_sync(FULL, g, j);
            if (((ip >> j) & 1u) && gj < g) ++rank;
        }
        if (inprog) {
            park = rank;
            s_len[w][rank] = rem;
            s_src[w][rank] = cur;
            s_row[w][rank] = row;
        }
        const int n_un = nrows - next_g;
        ntail = n_in + n_un;  // <= 62 by construction
        for (int j = lane; j < n_un; j += 32) {
            const int r = r_first + next_g + j;
            const int a = arp[r], bb = arp[r + 1];
            s_len[w][n_in + j] = (int)(((long long)bb < e ? bb : e) - a);
            s_src[w][n_in + j] = a;
            s_row[w][n_in + j] = r;
        }
        __syncwarp();
        const int l0 = lane < ntail ? s_len[w][lane] : 0;
        const int l1 = lane + 32 < ntail ? s_len[w][lane + 32] : 0;
        const int e0 = warp_excl_scan(l0, lane);
        const int tot0 = __shfl_sync(FULL, e0 + l0, 31);
        const int e1 = warp_excl_scan(l1, lane) + tot0;
        if (lane < ntail) s_off[w][lane] = e0;
        if (lane + 32 < ntail) s_off[w][lane + 32] = e1;
        __syncwarp();
        // lane's share of the tail: concatenation positions [lane*T, lane*T + T)
        const int pos = lane * T;
        int lo = 0, hi = ntail;  // last slot j with s_off[j] <= pos
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_off[w][mid] <= pos) lo = mid; else hi = mid;
        }
        int j = lo;
        int off = pos - s_off[w][j];
        first_slot = j;
        contm = __ballot_sync(FULL, off != 0);
        int slen = s_len[w][j], sa = s_src[w][j];
        src = row_src(rp, arp, m, s_row[w][j]);
        for (int t = 0; t < T; ++t, ++i) {
            put_elem<VT, IT>(vals, cols, s, i, lane, ci, v, sa + off, src, col_base, ovf);
            ++off;
            const bool slot_end = (off == slen);
            if (slot_end || t == T - 1) fword |= 1u << (i & 31);
            if ((i & 31) == 31) { fb[(i >> 5) * 32 + lane] = fword; fword = 0; }
            if (slot_end && t + 1 < T) {
                ++j;
                off = 0;
                slen = s_len[w][j];
                sa = s_src[w][j];
                src = row_src(rp, arp, m, s_row[w][j]);
            }
        }
    }
    CvrMeta *M = meta + c;
    if (lane == 0) {
        unsigned sh = 0;
        if ((long long)arp[r_first] < s) sh |= 1u;
        if ((long long)arp[r_last + 1] > e) sh |= 2u;
        M->h.r_first = r_first;
        M->h.nrows = nrows;
        M->h.shared = sh;
        M->h.aux = 0;
        M->i_t = i_t;
        M->ntail = ntail;
        M->n_inprog = n_in;
        M->next_g = next_g;
        M->cont = contm;
    }
    M->park[lane] = (unsigned char)park;
    M->first_slot[lane] = (unsigned char)first_slot;
}

// ---------------------------------------------------------------------------------------
// CVR SpMV.  One warp per chunk (grid-stride).  The chunk is walked in 4-step blocks with a
// software pipeline: value and flag streams are requested two blocks ahead, column streams
// three blocks ahead, and the x gathers one block ahead of the block being summed, so each
// lane keeps several 16-byte stream loads and four gathers in flight.
#ifndef PAVA_CVR_MINB32
#define PAVA_CVR_MINB32 3
#endif
#ifndef PAVA_CVR_MINB
#define PAVA_CVR_MINB 2
#endif
constexpr int SPMV_WARPS = 8;

template <int S, typename VT, typename IT>
__global__ void __launch_bounds__(SPMV_WARPS * 32, sizeof(VT) == 8 ? PAVA_CVR_MINB : PAVA_CVR_MINB32)
cvr_spmv_kernel(const CvrMeta *__restrict__ meta, const unsigned *__restrict__ flags,
                const VT *__restrict__ vals, const IT *__restrict__ cols,
                const VT *__restrict__ x, const int *__restrict__ colbase,
                double *__restrict__ y, double *__restrict__ carry_head,
                double *__restrict__ carry_tail, long long nchunks, int m, int n,
                unsigned long long *err) {
    constexpr int L = 32 * S;
    constexpr int NB = S / 4;
    __shared__ double s_tail[SPMV_WARPS][64];
    __shared__ int s_row[SPMV_WARPS][64];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
    const unsigned lt = lanemask_lt();
    // the carry fixup that follows may launch now; it waits for this grid to finish
    asm volatile("griddepcontrol.launch_dependents;");
    const long long nwarps = (long long)gridDim.x * SPMV_WARPS;

    for (long long c = (long long)blockIdx.x * SPMV_WARPS + w; c < nchunks; c += nwarps) {
        const CvrMeta *M = meta + c;
        const int r_first = M->h.r_first;
        const int r_last = r_first + M->h.nrows - 1;
        const unsigned shared = M->h.shared;
        const int i_t = M->i_t;
        const VT *vb = vals + c * L;
        const IT *cb = cols + c * L;
        const int xbase = sizeof(IT) == 2 ? colbase[c] : 0;  // base of the column offsets
        const VT *xb = x + xbase;
        const int xlo = -xbase, xhi = n - xbase;  // the offsets that stay inside x
        const unsigned *fb = flags + c * S;
        auto LF = [&](int b) { return ld_flag(fb + ((4 * b) >> 5) * 32 + lane); };

        Acc<VT> acc;
        int g = lane, next_g = 32;
        int slot = 0, nfrag = 0, last_nfrag = 0;
        bool cont = false;
        double cin = 0.0, last = 0.0;

        // prologue: x of block 0, values/flags of blocks 0-1, columns of blocks 1-2
        CBlk<IT> c1 = CBlk<IT>::load(cb, 1, lane, pf), c2 = CBlk<IT>::load(cb, 2, lane, pf);
        VBlk<VT> v0 = VBlk<VT>::load(vb, 0, lane, pf), v1 = VBlk<VT>::load(vb, 1, lane, pf);
        unsigned f0 = LF(0), f1 = LF(1);
        VT x0[4];
        {
            const CBlk<IT> c0 = CBlk<IT>::load(cb, 0, lane, pf);
#pragma unroll
            for (int q = 0; q < 4; ++q) x0[q] = c0.gather(q, xb, pl, xlo, xhi, err);
        }
#pragma unroll 1
        for (int blk = 0; blk < NB; ++blk) {
            CBlk<IT> cn = c2;
            VBlk<VT> vn = v1;
            unsigned fn = f1;
            if (blk + 3 < NB) cn = CBlk<IT>::load(cb, blk + 3, lane, pf);
            if (blk + 2 < NB) {
                vn = VBlk<VT>::load(vb, blk + 2, lane, pf);
                fn = LF(blk + 2);
            }
            VT x1[4];
            if (blk + 1 < NB) {
#pragma unroll
                for (int q = 0; q < 4; ++q) x1[q] = c1.gather(q, xb, pl, xlo, xhi, err);
            }
            const unsigned fw = f0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int i = blk * 4 + q;
                const bool f = (fw >> (i & 31)) & 1u;
                if (i < i_t) {
                    acc.add(v0.get(q), x0[q]);
                    const unsigned bal = __ballot_sync(FULL, f);
                    if (f) {
                        flush_row(r_first + g, acc.value(), r_first, r_last, shared, c, y,
                                  carry_head, carry_tail, m, err);
                        acc.reset();
                        g = next_g + __popc(bal & lt);
                    }
                    next_g += __popc(bal);
                } else {
                    if (i == i_t) {  // tail start: park the open rows' partial sums
                        s_tail[w][lane] = 0.0;
                        s_tail[w][lane + 32] = 0.0;
                        __syncwarp();
                        const int pk = M->park[lane];
                        if (pk != 0xff && guard(err, pk < 64, G_SLOT, pk)) {
                            s_tail[w][pk] = acc.value();
                            s_row[w][pk] = r_first + g;
                        }
                        acc.reset();
                        slot = M->first_slot[lane];
                        cont = (M->cont >> lane) & 1u;
                        nfrag = 0;
                        __syncwarp();
                    }
                    acc.add(v0.get(q), x0[q]);
                    if (f) {
                        const double a = acc.value();
                        if (i == S - 1) { last = a; last_nfrag = nfrag; }
                        else if (nfrag == 0 && cont) cin = a;
                        else if (guard(err, slot >= 0 && slot < 64, G_SLOT, slot))
                            s_tail[w][slot] += a;  // a fragment that starts in this lane
                        ++slot;
                        ++nfrag;
                        acc.reset();
                    }
                }
            }
            c1 = c2; c2 = cn;
            v0 = v1; v1 = vn;
            f0 = f1; f1 = fn;
#pragma unroll
            for (int q = 0; q < 4; ++q) x0[q] = x1[q];
        }
        if (i_t < S) {
            // combine fragments that continue across lanes, then store the tail rows
            const unsigned contm = M->cont;
            const bool single = (last_nfrag == 0);
            const bool link = lane < 31 && ((contm >> (lane + 1)) & 1u);
            const double a = (single && cont) ? last : (cont ? cin : 0.0);
            const double H = seg_suffix(a, single && cont && link, lane);
            const double Hn = __shfl_down_sync(FULL, H, 1);
            if (!(single && cont) && guard(err, slot >= 1 && slot <= 64, G_SLOT, slot - 1))
                s_tail[w][slot - 1] += last + (link ? Hn : 0.0);
            __syncwarp();
            int ntail = M->ntail, n_in = M->n_inprog;
            const int ng = M->next_g;
            if (!guard(err, ntail >= 0 && ntail <= 64 && n_in >= 0 && n_in <= ntail, G_SLOT,
                       ntail))
                ntail = n_in = 0;
            for (int j = lane; j < ntail; j += 32) {
                const int row = j < n_in ? s_row[w][j] : r_first + ng + (j - n_in);
                flush_row(row, s_tail[w][j], r_first, r_last, shared, c, y, carry_head,
                          carry_tail, m, err);
            }
            __syncwarp();
        }
    }
}

template <typename VT, typename IT>
cudaError_t convert_t(Handle &h, const int *rp, const int *ci, const double *v, int *ovf,
                      cudaStream_t s) {
    const long long blocks = (h.nchunks + CONV_WARPS - 1) / CONV_WARPS;
    cvr_convert_kernel<VT, IT><<<(unsigned)blocks, CONV_WARPS * 32, 0, s>>>(
        rp, ci, v, h.arp, h.m, h.nchunks, h.S, (VT *)h.vals, (IT *)h.cols, h.flags,
        (CvrMeta *)h.meta, h.colbase, ovf);
    return cudaGetLastError();
}

template <typename VT, typename IT>
cudaError_t spmv_t(const Handle &h, const void *x, void *y, cudaStream_t s) {
    const long long want = (h.nchunks + SPMV_WARPS - 1) / SPMV_WARPS;
    const long long cap = (long long)h.sm_count * (sizeof(VT) == 8 ? PAVA_CVR_MINB : PAVA_CVR_MINB32);
    const unsigned grid = (unsigned)(want < cap ? want : cap);
    const CvrMeta *meta = (const CvrMeta *)h.meta;
    const VT *xv = (const VT *)x;
    double *yv = (double *)y;
    switch (h.S) {
        case 32:
            cvr_spmv_kernel<32, VT, IT><<<grid, SPMV_WARPS * 32, 0, s>>>(
                meta, h.flags, (const VT *)h.vals, (const IT *)h.cols, xv, h.colbase, yv,
                h.carry_head, h.carry_tail, h.nchunks, h.m, h.n, guard_word());
            break;
        case 64:
            cvr_spmv_kernel<64, VT, IT><<<grid, SPMV_WARPS * 32, 0, s>>>(
                meta, h.flags, (const VT *)h.vals, (const IT *)h.cols, xv, h.colbase, yv,
                h.carry_head, h.carry_tail, h.nchunks, h.m, h.n, guard_word());
            break;
        case 128:
            cvr_spmv_kernel<128, VT, IT><<<grid, SPMV_WARPS * 32, 0, s>>>(
                meta, h.flags, (const VT *)h.vals, (const IT *)h.cols, xv, h.colbase, yv,
                h.carry_head, h.carry_tail, h.nchunks, h.m, h.n, guard_word());
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t cvr_convert(Handle &h, const int *rp, const int *ci, const double *v, int *ovf,
                        cudaStream_t s) {
    if (h.nchunks <= 0) return cudaSuccess;
    const bool f32 = h.precision == PAVA_PREC_FP32C, d16 = h.index_mode == PAVA_INDEX_DELTA16;
    if (!f32 && !d16) return convert_t<double, int>(h, rp, ci, v, ovf, s);
    if (!f32 && d16) return convert_t<double, short>(h, rp, ci, v, ovf, s);
    if (f32 && !d16) return convert_t<float, int>(h, rp, ci, v, ovf, s);
    return convert_t<float, short>(h, rp, ci, v, ovf, s);
}

cudaError_t cvr_spmv(const Handle &h, const void *x, void *y, cudaStream_t s) {
    if (h.nchunks <= 0) return cudaSuccess;
    const bool f32 = h.precision == PAVA_PREC_FP32C, d16 = h.index_mode == PAVA_INDEX_DELTA16;
    if (!f32 && !d16) return spmv_t<double, int>(h, x, y, s);
    if (!f32 && d16) return spmv_t<double, short>(h, x, y, s);
    if (f32 && !d16) return spmv_t<float, int>(h, x, y, s);
    return spmv_t<float, short>(h, x, y, s);
}

}  // namespace pava
