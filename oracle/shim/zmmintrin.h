/*
 * Test infrastructure (oracle only): maps the Knights-Corner/KNL spellings of six AVX-512
 * intrinsics that the reference engines use onto their AVX-512F names, so that GCC can
 * compile the reference's cvr/cvr.h and csr5/anonymouslib_avx512.h unchanged on an
 * AVX-512 host.  The reference's csr5/detail/avx512/common_avx512.h:7 includes
 * "zmmintrin.h"; this file is what that include resolves to.
 *
 *   _mm512_i32logather_pd       -> gather 8 doubles with the low 8 int32 indices
 *   _mm512_(mask_)i32loscatter_pd -> scatter 8 doubles with the low 8 int32 indices
 *   _mm512_permute4f128_epi32    -> 128-bit lane shuffle (same imm8 encoding)
 *   _mm512_permutevar_epi32      -> full int32 permute (index operand first)
 *   _MM_SCALE_8 / _MM_SCALE_4    -> literal gather scales
 */
#ifndef PAVA_ORACLE_KNC_SHIM_H
#define PAVA_ORACLE_KNC_SHIM_H

#include <immintrin.h>

#define _MM_SCALE_8 8
#define _MM_SCALE_4 4

#define _mm512_i32logather_pd(idx, base, scale) \
    _mm512_i32gather_pd(_mm512_castsi512_si256(idx), (base), (scale))
#define _mm512_mask_i32loscatter_pd(base, k, idx, v, scale) \
    _mm512_mask_i32scatter_pd((base), (k), _mm512_castsi512_si256(idx), (v), (scale))
#define _mm512_i32loscatter_pd(base, idx, v, scale) \
    _mm512_i32scatter_pd((base), _mm512_castsi512_si256(idx), (v), (scale))
#define _mm512_permute4f128_epi32(v, perm) _mm512_shuffle_i32x4((v), (v), (perm))
#define _mm512_permutevar_epi32(idx, v) _mm512_permutexvar_epi32((idx), (v))

#endif
