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
//    reference's (position, row) records): the SpMV stores the lane's FMA accumulator into y
//    there.  Rows a lane finishes are summed in CSR order, one FMA per element.
//  * tail: when a lane finishes and no row is left to take, the rest of the chunk -- the open
//    rows' remaining elements, in row order -- is spread evenly over the 32 lanes (the GPU
//    form of the reference's stealing).  Partial sums meet in shared memory through a
//    fixed-order segmented suffix scan, so the result does not depend on timing.
//  * a chunk's first / last row may continue in the neighbouring chunk; their partial sums go
//    to per-chunk carry slots that k_fixup.cu adds in chunk order (the reference adds them
//    with `omp atomic`, cvr/cvr.h:1415,1717,1855).
//
// Empty rows are given one element of value 0 in column -1 (which reads no x), so that every
// row is visited and written: y = A x overwrites all of y on every call.  The last chunk is
// padded with such elements, which belong to a padding row m whose sum is dropped.
//
// Layout of chunk c (L = 32*S elements, element (step i, lane k)):
//   values  at c*L + (i/VP)*32*VP + VP*k + i%VP   (VP values per 16-byte lane load)
//   columns at c*L + (i/CP)*32*CP + CP*k + i%CP   (CP columns per 16-byte lane load)
//   flags   word w of lane k at c*S + 32*w + k, bit i%32 of word i/32

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

template <int VP, int CP, typename VT>
__device__ __forceinline__ void put_elem(VT *vals, int *cols, long long cbase, int i, int lane,
                                         const int *ci, const double *v, int e, RowSrc src) {
    double val = 0.0;
    int col = -1;
    if (!src.dummy) {
        val = v[e + src.base];
        col = ci[e + src.base];
    }
    vals[cbase + (i / VP) * 32 * VP + VP * lane + (i % VP)] = (VT)val;
    cols[cbase + (i / CP) * 32 * CP + CP * lane + (i % CP)] = col;
}

constexpr int CONV_WARPS = 4;

template <int VP, int CP, typename VT>
__global__ void __launch_bounds__(CONV_WARPS * 32)
cvr_convert_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                   const double *__restrict__ v, const int *__restrict__ arp, int m,
                   long long nchunks, int S, VT *__restrict__ vals, int *__restrict__ cols,
                   unsigned *__restrict__ flags, CvrMeta *__restrict__ meta) {
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
        put_elem<VP, CP>(vals, cols, s, i, lane, ci, v, cur, src);
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
            put_elem<VP, CP>(vals, cols, s, i, lane, ci, v, sa + off, src);
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
// CVR SpMV, FP64.  One warp per chunk (grid-stride), 8 steps per loop trip: two int4 column
// loads, four double2 value loads and one flag word per lane, with the next trip's streams
// requested before this trip's x gathers are consumed.
constexpr int SPMV_WARPS = 8;

template <int S>
__global__ void __launch_bounds__(SPMV_WARPS * 32)
cvr_spmv_f64_kernel(const CvrMeta *__restrict__ meta, const unsigned *__restrict__ flags,
                    const double *__restrict__ vals, const int *__restrict__ cols,
                    const double *__restrict__ x, double *__restrict__ y,
                    double *__restrict__ carry_head, double *__restrict__ carry_tail,
                    long long nchunks, int m) {
    constexpr int L = 32 * S;
    constexpr int NB = S / 8;
    __shared__ double s_tail[SPMV_WARPS][64];
    __shared__ int s_row[SPMV_WARPS][64];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
    const unsigned lt = lanemask_lt();
    const long long nwarps = (long long)gridDim.x * SPMV_WARPS;

    for (long long c = (long long)blockIdx.x * SPMV_WARPS + w; c < nchunks; c += nwarps) {
        const CvrMeta *M = meta + c;
        const int r_first = M->h.r_first;
        const int r_last = r_first + M->h.nrows - 1;
        const unsigned shared = M->h.shared;
        const int i_t = M->i_t;
        const double2 *vb = reinterpret_cast<const double2 *>(vals + c * L);
        const int4 *cb = reinterpret_cast<const int4 *>(cols + c * L);
        const unsigned *fb = flags + c * S;

        double acc = 0.0;
        int g = lane, next_g = 32;
        int slot = 0, nfrag = 0, last_nfrag = 0;
        bool cont = false;
        double cin = 0.0, last = 0.0;

        int4 c0 = ld_stream(cb + lane, pf), c1 = ld_stream(cb + 32 + lane, pf);
        double2 v0 = ld_stream(vb + lane, pf), v1 = ld_stream(vb + 32 + lane, pf);
        double2 v2 = ld_stream(vb + 64 + lane, pf), v3 = ld_stream(vb + 96 + lane, pf);
        unsigned fw = ld_stream(fb + lane, pf);
#pragma unroll 1
        for (int blk = 0; blk < NB; ++blk) {
            const int i0 = blk * 8;
            int4 nc0, nc1;
            double2 nv0, nv1, nv2, nv3;
            unsigned nfw = fw;
            if (blk + 1 < NB) {
                nc0 = ld_stream(cb + (2 * blk + 2) * 32 + lane, pf);
                nc1 = ld_stream(cb + (2 * blk + 3) * 32 + lane, pf);
                nv0 = ld_stream(vb + (4 * blk + 4) * 32 + lane, pf);
                nv1 = ld_stream(vb + (4 * blk + 5) * 32 + lane, pf);
                nv2 = ld_stream(vb + (4 * blk + 6) * 32 + lane, pf);
                nv3 = ld_stream(vb + (4 * blk + 7) * 32 + lane, pf);
                if (((i0 + 8) & 31) == 0) nfw = ld_stream(fb + ((i0 + 8) >> 5) * 32 + lane, pf);
            }
            const int cc[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
            const double vv[8] = {v0.x, v0.y, v1.x, v1.y, v2.x, v2.y, v3.x, v3.y};
            double xx[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) xx[q] = gather_x(x, cc[q], pl);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int i = i0 + q;
                const bool f = (fw >> (i & 31)) & 1u;
                if (i < i_t) {
                    acc = fma(vv[q], xx[q], acc);
                    const unsigned bal = __ballot_sync(FULL, f);
                    if (f) {
                        flush_row(r_first + g, acc, r_first, r_last, shared, c, y, carry_head,
                                  carry_tail, m);
                        acc = 0.0;
                        g = next_g + __popc(bal & lt);
                    }
                    next_g += __popc(bal);
                } else {
                    if (i == i_t) {  // tail start: park the open rows' partial sums
                        s_tail[w][lane] = 0.0;
                        s_tail[w][lane + 32] = 0.0;
                        __syncwarp();
                        const int pk = M->park[lane];
                        if (pk != 0xff) {
                            s_tail[w][pk] = acc;
                            s_row[w][pk] = r_first + g;
                        }
                        acc = 0.0;
                        slot = M->first_slot[lane];
                        cont = (M->cont >> lane) & 1u;
                        nfrag = 0;
                        __syncwarp();
                    }
                    acc = fma(vv[q], xx[q], acc);
                    if (f) {
                        if (i == S - 1) { last = acc; last_nfrag = nfrag; }
                        else if (nfrag == 0 && cont) cin = acc;
                        else s_tail[w][slot] += acc;  // a fragment that starts in this lane
                        ++slot;
                        ++nfrag;
                        acc = 0.0;
                    }
                }
            }
            c0 = nc0; c1 = nc1;
            v0 = nv0; v1 = nv1; v2 = nv2; v3 = nv3;
            fw = nfw;
        }
        if (i_t < S) {
            // combine fragments that continue across lanes, then store the tail rows
            const unsigned contm = M->cont;
            const bool single = (last_nfrag == 0);
            const bool link = lane < 31 && ((contm >> (lane + 1)) & 1u);
            const double a = (single && cont) ? last : (cont ? cin : 0.0);
            const double H = seg_suffix(a, single && cont && link, lane);
            const double Hn = __shfl_down_sync(FULL, H, 1);
            if (!(single && cont)) s_tail[w][slot - 1] += last + (link ? Hn : 0.0);
            __syncwarp();
            const int ntail = M->ntail, n_in = M->n_inprog, ng = M->next_g;
            for (int j = lane; j < ntail; j += 32) {
                const int row = j < n_in ? s_row[w][j] : r_first + ng + (j - n_in);
                flush_row(row, s_tail[w][j], r_first, r_last, shared, c, y, carry_head,
                          carry_tail, m);
            }
            __syncwarp();
        }
    }
}

}  // namespace

cudaError_t cvr_convert(Handle &h, const int *rp, const int *ci, const double *v,
                        cudaStream_t s) {
    const long long blocks = (h.nchunks + CONV_WARPS - 1) / CONV_WARPS;
    if (blocks <= 0) return cudaSuccess;
    if (h.precision == PAVA_PREC_FP64) {
        cvr_convert_kernel<2, 4, double><<<(unsigned)blocks, CONV_WARPS * 32, 0, s>>>(
            rp, ci, v, h.arp, h.m, h.nchunks, h.S, (double *)h.vals, (int *)h.cols, h.flags,
            (CvrMeta *)h.meta);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t cvr_spmv(const Handle &h, const void *x, void *y, cudaStream_t s) {
    if (h.nchunks <= 0) return cudaSuccess;
    const long long want = (h.nchunks + SPMV_WARPS - 1) / SPMV_WARPS;
    const long long cap = (long long)h.sm_count * 8;
    const unsigned grid = (unsigned)(want < cap ? want : cap);
    if (h.precision != PAVA_PREC_FP64) return cudaErrorInvalidValue;
#define PAVA_CVR_LAUNCH(SV)                                                                 \
    cvr_spmv_f64_kernel<SV><<<grid, SPMV_WARPS * 32, 0, s>>>(                               \
        (const CvrMeta *)h.meta, h.flags, (const double *)h.vals, (const int *)h.cols,      \
        (const double *)x, (double *)y, h.carry_head, h.carry_tail, h.nchunks, h.m)
    switch (h.S) {
        case 32: PAVA_CVR_LAUNCH(32); break;
        case 64: PAVA_CVR_LAUNCH(64); break;
        case 128: PAVA_CVR_LAUNCH(128); break;
        default: return cudaErrorInvalidValue;
    }
#undef PAVA_CVR_LAUNCH
    return cudaGetLastError();
}

}  // namespace pava
