/* vectormath_hyp_avx512.h -- AVX-512 forms of the shared tanh / atanh
 * (simd-fecfun_b200/csrc/ldpc_math.h) for 16 floats and 8 doubles, for the
 * reference's sum-product builds (oracle / CPU-baseline only).
 *
 * Every lane runs exactly the scalar functions' operations, in the same
 * order: correctly rounded +, -, *, / and fused multiply-adds, the same
 * constants, the same round-to-nearest trick and exponent arithmetic.  Where
 * the scalar code branches, both sides are computed for all lanes and the
 * lane's own side is selected, so each lane's result is the scalar result
 * bit for bit.
 */
#ifndef VCL_COMPAT_VECTORMATH_HYP_AVX512_H
#define VCL_COMPAT_VECTORMATH_HYP_AVX512_H
#if defined(__AVX512F__) && defined(__AVX512DQ__)
#include <immintrin.h>

/* ---------------- float x 16 ---------------- */
static inline __m512 vlm_fma(__m512 a, __m512 b, __m512 c) { return _mm512_fmadd_ps(a, b, c); }
static inline __m512 vlm_c(float v) { return _mm512_set1_ps(v); }

static inline __m512 vlm_rint(__m512 x) {
    const __m512 magic = vlm_c(12582912.0f);
    return _mm512_sub_ps(_mm512_add_ps(x, magic), magic);
}

static inline __m512 vlm_exp_neg(__m512 y) {
    __m512 k = vlm_rint(_mm512_mul_ps(y, vlm_c(1.44269502162933349609375f)));
    const __m512 nk = _mm512_castsi512_ps(_mm512_xor_si512(_mm512_castps_si512(k), _mm512_set1_epi32((int)0x80000000u)));
    __m512 r = vlm_fma(nk, vlm_c(1.428606765330187045e-06f), vlm_fma(nk, vlm_c(0.693145751953125f), y));
    __m512 p = vlm_c(2.4801587301587302e-05f);
    p = vlm_fma(p, r, vlm_c(1.9841269841269841e-04f));
    p = vlm_fma(p, r, vlm_c(1.3888888888888889e-03f));
    p = vlm_fma(p, r, vlm_c(8.3333333333333333e-03f));
    p = vlm_fma(p, r, vlm_c(4.1666666666666667e-02f));
    p = vlm_fma(p, r, vlm_c(1.6666666666666667e-01f));
    p = vlm_fma(p, r, vlm_c(0.5f));
    p = vlm_fma(p, r, vlm_c(1.0f));
    p = vlm_fma(p, r, vlm_c(1.0f));
    const __m512i ki = _mm512_cvttps_epi32(k);
    const __m512 scale = _mm512_castsi512_ps(_mm512_slli_epi32(_mm512_add_epi32(ki, _mm512_set1_epi32(127)), 23));
    return _mm512_mul_ps(p, scale);
}

static inline __m512 vlm_expm1_neg(__m512 y) {
    __m512 p = vlm_c(2.7557319223985891e-06f);
    p = vlm_fma(p, y, vlm_c(2.4801587301587302e-05f));
    p = vlm_fma(p, y, vlm_c(1.9841269841269841e-04f));
    p = vlm_fma(p, y, vlm_c(1.3888888888888889e-03f));
    p = vlm_fma(p, y, vlm_c(8.3333333333333333e-03f));
    p = vlm_fma(p, y, vlm_c(4.1666666666666667e-02f));
    p = vlm_fma(p, y, vlm_c(1.6666666666666667e-01f));
    p = vlm_fma(p, y, vlm_c(0.5f));
    p = vlm_fma(p, y, vlm_c(1.0f));
    const __m512 small = _mm512_mul_ps(p, y);
    const __m512 big = _mm512_sub_ps(vlm_exp_neg(y), vlm_c(1.0f));
    const __mmask16 is_small = _mm512_cmp_ps_mask(y, vlm_c(-0.25f), _CMP_GT_OQ);
    return _mm512_mask_blend_ps(is_small, big, small);
}

static inline __m512 vlm_log_series(__m512 s) {
    const __m512 s2 = _mm512_mul_ps(s, s);
    __m512 p = vlm_c(7.6923076923076923e-02f);
    p = vlm_fma(p, s2, vlm_c(9.0909090909090909e-02f));
    p = vlm_fma(p, s2, vlm_c(1.1111111111111111e-01f));
    p = vlm_fma(p, s2, vlm_c(1.4285714285714286e-01f));
    p = vlm_fma(p, s2, vlm_c(2.0000000000000000e-01f));
    p = vlm_fma(p, s2, vlm_c(3.3333333333333333e-01f));
    p = vlm_fma(p, s2, vlm_c(1.0f));
    return _mm512_mul_ps(vlm_c(2.0f), _mm512_mul_ps(p, s));
}

static inline __m512 vlm_log1p_pos(__m512 t) {
    const __m512 small = vlm_log_series(_mm512_div_ps(t, _mm512_add_ps(vlm_c(2.0f), t)));
    const __m512 u = _mm512_add_ps(vlm_c(1.0f), t);
    const __m512i iu = _mm512_castps_si512(u);
    __m512i e = _mm512_sub_epi32(_mm512_and_si512(_mm512_srli_epi32(iu, 23), _mm512_set1_epi32(0xff)), _mm512_set1_epi32(127));
    __m512 f = _mm512_castsi512_ps(_mm512_or_si512(_mm512_and_si512(iu, _mm512_set1_epi32(0x007fffff)),
                                                   _mm512_set1_epi32(0x3f800000)));
    const __mmask16 hi = _mm512_cmp_ps_mask(f, vlm_c(1.41421356f), _CMP_GT_OQ);
    f = _mm512_mask_mul_ps(f, hi, f, vlm_c(0.5f));
    e = _mm512_mask_add_epi32(e, hi, e, _mm512_set1_epi32(1));
    const __m512 s = _mm512_div_ps(_mm512_sub_ps(f, vlm_c(1.0f)), _mm512_add_ps(f, vlm_c(1.0f)));
    const __m512 ef = _mm512_cvtepi32_ps(e);
    const __m512 corr = _mm512_div_ps(_mm512_sub_ps(t, _mm512_sub_ps(u, vlm_c(1.0f))), u);
    const __m512 lo = _mm512_add_ps(vlm_fma(ef, vlm_c(1.428606765330187045e-06f), vlm_log_series(s)), corr);
    const __m512 big = vlm_fma(ef, vlm_c(0.693145751953125f), lo);
    return _mm512_mask_blend_ps(_mm512_cmp_ps_mask(t, vlm_c(0.25f), _CMP_LT_OQ), big, small);
}

static inline __m512 vlm_tanh(__m512 x) {
    const __m512i sign = _mm512_set1_epi32((int)0x80000000u);
    const __m512 a = _mm512_castsi512_ps(_mm512_andnot_si512(sign, _mm512_castps_si512(x)));
    const __m512 e = vlm_expm1_neg(_mm512_mul_ps(vlm_c(-2.0f), a));
    __m512 r = _mm512_div_ps(_mm512_sub_ps(_mm512_setzero_ps(), e), _mm512_add_ps(vlm_c(2.0f), e));
    r = _mm512_mask_blend_ps(_mm512_cmp_ps_mask(a, vlm_c(10.0f), _CMP_LT_OQ), vlm_c(1.0f), r);
    return _mm512_castsi512_ps(_mm512_or_si512(_mm512_castps_si512(r), _mm512_and_si512(_mm512_castps_si512(x), sign)));
}

static inline __m512 vlm_atanh(__m512 m) {
    const __m512i sign = _mm512_set1_epi32((int)0x80000000u);
    const __m512 a = _mm512_castsi512_ps(_mm512_andnot_si512(sign, _mm512_castps_si512(m)));
    const __m512 t = _mm512_div_ps(_mm512_add_ps(a, a), _mm512_sub_ps(vlm_c(1.0f), a));
    const __m512 r = _mm512_mul_ps(vlm_c(0.5f), vlm_log1p_pos(t));
    return _mm512_castsi512_ps(_mm512_or_si512(_mm512_castps_si512(r), _mm512_and_si512(_mm512_castps_si512(m), sign)));
}

/* ---------------- double x 8 ---------------- */
static inline __m512d vlmd_fma(__m512d a, __m512d b, __m512d c) { return _mm512_fmadd_pd(a, b, c); }
static inline __m512d vlmd_c(double v) { return _mm512_set1_pd(v); }

static inline __m512d vlmd_rint(__m512d x) {
    const __m512d magic = vlmd_c(6755399441055744.0);
    return _mm512_sub_pd(_mm512_add_pd(x, magic), magic);
}

static inline __m512d vlmd_exp_neg(__m512d y) {
    __m512d k = vlmd_rint(_mm512_mul_pd(y, vlmd_c(1.4426950408889634)));
    const __m512d nk = _mm512_castsi512_pd(_mm512_xor_si512(_mm512_castpd_si512(k), _mm512_set1_epi64((long long)0x8000000000000000ULL)));
    __m512d r = vlmd_fma(nk, vlmd_c(LMD_LN2_LO), vlmd_fma(nk, vlmd_c(LMD_LN2_HI), y));
    __m512d p = vlmd_c(1.1470745597729725e-11);
    p = vlmd_fma(p, r, vlmd_c(1.6059043836821613e-10));
    p = vlmd_fma(p, r, vlmd_c(2.08767569878681e-09));
    p = vlmd_fma(p, r, vlmd_c(2.505210838544172e-08));
    p = vlmd_fma(p, r, vlmd_c(2.7557319223985888e-07));
    p = vlmd_fma(p, r, vlmd_c(2.7557319223985893e-06));
    p = vlmd_fma(p, r, vlmd_c(2.4801587301587302e-05));
    p = vlmd_fma(p, r, vlmd_c(1.9841269841269841e-04));
    p = vlmd_fma(p, r, vlmd_c(1.3888888888888889e-03));
    p = vlmd_fma(p, r, vlmd_c(8.3333333333333332e-03));
    p = vlmd_fma(p, r, vlmd_c(4.1666666666666664e-02));
    p = vlmd_fma(p, r, vlmd_c(1.6666666666666666e-01));
    p = vlmd_fma(p, r, vlmd_c(0.5));
    p = vlmd_fma(p, r, vlmd_c(1.0));
    p = vlmd_fma(p, r, vlmd_c(1.0));
    const __m512i ki = _mm512_cvttpd_epi64(k);
    const __m512d scale = _mm512_castsi512_pd(_mm512_slli_epi64(_mm512_add_epi64(ki, _mm512_set1_epi64(1023)), 52));
    return _mm512_mul_pd(p, scale);
}

static inline __m512d vlmd_expm1_neg(__m512d y) {
    __m512d p = vlmd_c(1.1470745597729725e-11);
    p = vlmd_fma(p, y, vlmd_c(1.6059043836821613e-10));
    p = vlmd_fma(p, y, vlmd_c(2.08767569878681e-09));
    p = vlmd_fma(p, y, vlmd_c(2.505210838544172e-08));
    p = vlmd_fma(p, y, vlmd_c(2.7557319223985888e-07));
    p = vlmd_fma(p, y, vlmd_c(2.7557319223985893e-06));
    p = vlmd_fma(p, y, vlmd_c(2.4801587301587302e-05));
    p = vlmd_fma(p, y, vlmd_c(1.9841269841269841e-04));
    p = vlmd_fma(p, y, vlmd_c(1.3888888888888889e-03));
    p = vlmd_fma(p, y, vlmd_c(8.3333333333333332e-03));
    p = vlmd_fma(p, y, vlmd_c(4.1666666666666664e-02));
    p = vlmd_fma(p, y, vlmd_c(1.6666666666666666e-01));
    p = vlmd_fma(p, y, vlmd_c(0.5));
    p = vlmd_fma(p, y, vlmd_c(1.0));
    const __m512d small = _mm512_mul_pd(p, y);
    const __m512d big = _mm512_sub_pd(vlmd_exp_neg(y), vlmd_c(1.0));
    return _mm512_mask_blend_pd(_mm512_cmp_pd_mask(y, vlmd_c(-0.25), _CMP_GT_OQ), big, small);
}

static inline __m512d vlmd_log_series(__m512d s) {
    const __m512d s2 = _mm512_mul_pd(s, s);
    __m512d p = vlmd_c(0.040000000000000001);
    p = vlmd_fma(p, s2, vlmd_c(0.043478260869565216));
    p = vlmd_fma(p, s2, vlmd_c(0.047619047619047616));
    p = vlmd_fma(p, s2, vlmd_c(0.052631578947368418));
    p = vlmd_fma(p, s2, vlmd_c(0.058823529411764705));
    p = vlmd_fma(p, s2, vlmd_c(0.066666666666666666));
    p = vlmd_fma(p, s2, vlmd_c(0.076923076923076927));
    p = vlmd_fma(p, s2, vlmd_c(0.090909090909090912));
    p = vlmd_fma(p, s2, vlmd_c(0.1111111111111111));
    p = vlmd_fma(p, s2, vlmd_c(0.14285714285714285));
    p = vlmd_fma(p, s2, vlmd_c(0.20000000000000001));
    p = vlmd_fma(p, s2, vlmd_c(0.33333333333333331));
    p = vlmd_fma(p, s2, vlmd_c(1.0));
    return _mm512_mul_pd(vlmd_c(2.0), _mm512_mul_pd(p, s));
}

static inline __m512d vlmd_log1p_pos(__m512d t) {
    const __m512d small = vlmd_log_series(_mm512_div_pd(t, _mm512_add_pd(vlmd_c(2.0), t)));
    const __m512d u = _mm512_add_pd(vlmd_c(1.0), t);
    const __m512i iu = _mm512_castpd_si512(u);
    __m512i e = _mm512_sub_epi64(_mm512_and_si512(_mm512_srli_epi64(iu, 52), _mm512_set1_epi64(0x7ff)), _mm512_set1_epi64(1023));
    __m512d f = _mm512_castsi512_pd(_mm512_or_si512(_mm512_and_si512(iu, _mm512_set1_epi64(0x000fffffffffffffLL)),
                                                    _mm512_set1_epi64(0x3ff0000000000000LL)));
    const __mmask8 hi = _mm512_cmp_pd_mask(f, vlmd_c(1.4142135623730951), _CMP_GT_OQ);
    f = _mm512_mask_mul_pd(f, hi, f, vlmd_c(0.5));
    e = _mm512_mask_add_epi64(e, hi, e, _mm512_set1_epi64(1));
    const __m512d s = _mm512_div_pd(_mm512_sub_pd(f, vlmd_c(1.0)), _mm512_add_pd(f, vlmd_c(1.0)));
    const __m512d ef = _mm512_cvtepi64_pd(e);
    const __m512d corr = _mm512_div_pd(_mm512_sub_pd(t, _mm512_sub_pd(u, vlmd_c(1.0))), u);
    const __m512d lo = _mm512_add_pd(vlmd_fma(ef, vlmd_c(LMD_LN2_LO), vlmd_log_series(s)), corr);
    const __m512d big = vlmd_fma(ef, vlmd_c(LMD_LN2_HI), lo);
    return _mm512_mask_blend_pd(_mm512_cmp_pd_mask(t, vlmd_c(0.25), _CMP_LT_OQ), big, small);
}

static inline __m512d vlmd_tanh(__m512d x) {
    const __m512i sign = _mm512_set1_epi64((long long)0x8000000000000000ULL);
    const __m512d a = _mm512_castsi512_pd(_mm512_andnot_si512(sign, _mm512_castpd_si512(x)));
    const __m512d e = vlmd_expm1_neg(_mm512_mul_pd(vlmd_c(-2.0), a));
    __m512d r = _mm512_div_pd(_mm512_sub_pd(_mm512_setzero_pd(), e), _mm512_add_pd(vlmd_c(2.0), e));
    r = _mm512_mask_blend_pd(_mm512_cmp_pd_mask(a, vlmd_c(20.0), _CMP_LT_OQ), vlmd_c(1.0), r);
    return _mm512_castsi512_pd(_mm512_or_si512(_mm512_castpd_si512(r), _mm512_and_si512(_mm512_castpd_si512(x), sign)));
}

static inline __m512d vlmd_atanh(__m512d m) {
    const __m512i sign = _mm512_set1_epi64((long long)0x8000000000000000ULL);
    const __m512d a = _mm512_castsi512_pd(_mm512_andnot_si512(sign, _mm512_castpd_si512(m)));
    const __m512d t = _mm512_div_pd(_mm512_add_pd(a, a), _mm512_sub_pd(vlmd_c(1.0), a));
    const __m512d r = _mm512_mul_pd(vlmd_c(0.5), vlmd_log1p_pos(t));
    return _mm512_castsi512_pd(_mm512_or_si512(_mm512_castpd_si512(r), _mm512_and_si512(_mm512_castpd_si512(m), sign)));
}

#endif
#endif
