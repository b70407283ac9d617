/* vectormath_hyp.h -- compatibility header (oracle / CPU-baseline only).
 *
 * The reference's sum-product tree (src/LDPCDec/min_find.pl:37-48,98-106)
 * calls tanh() and atanh() on float (and double) vectors from vectorclass's
 * vectormath_hyp.h, which is absent here.  Both are mapped onto the
 * project's shared functions (simd-fecfun_b200/csrc/ldpc_math.h) -- lane by
 * lane, or for 16 floats / 8 doubles by their AVX-512 forms in
 * vectormath_hyp_avx512.h, bit-identical per lane --
 * the same code the GPU decoder runs, so the CPU oracle and the GPU agree
 * bit for bit.  This pins parity to that function, not to vectorclass's.
 */
#ifndef VCL_COMPAT_VECTORMATH_HYP_H
#define VCL_COMPAT_VECTORMATH_HYP_H
#include "vectorclass.h"
#include "ldpc_math.h"
#include "vectormath_hyp_avx512.h"

template <class V> static inline V vclc_lanewise(const V& a, float (*f)(float)) {
    V r;
    for (int i = 0; i < V::size(); ++i) r.e[i] = f(a.e[i]);
    return r;
}
static inline Vec8f tanh(const Vec8f a) { return vclc_lanewise(a, lm_tanh); }
static inline Vec16f tanh(const Vec16f a) {
#if defined(__AVX512F__) && defined(__AVX512DQ__)
    Vec16f r; _mm512_storeu_ps(r.e, vlm_tanh(_mm512_loadu_ps(a.e))); return r;
#else
    return vclc_lanewise(a, lm_tanh);
#endif
}
static inline Vec8f atanh(const Vec8f a) { return vclc_lanewise(a, lm_atanh); }
static inline Vec16f atanh(const Vec16f a) {
#if defined(__AVX512F__) && defined(__AVX512DQ__)
    Vec16f r; _mm512_storeu_ps(r.e, vlm_atanh(_mm512_loadu_ps(a.e))); return r;
#else
    return vclc_lanewise(a, lm_atanh);
#endif
}
/* double lanes (the SIMD_ELEM_BW=-64 builds): the shared double functions */
template <class V> static inline V vclc_lanewise_d(const V& a, double (*f)(double)) {
    V r;
    for (int i = 0; i < V::size(); ++i) r.e[i] = f(a.e[i]);
    return r;
}
static inline Vec4d tanh(const Vec4d a) { return vclc_lanewise_d(a, lmd_tanh); }
static inline Vec8d tanh(const Vec8d a) {
#if defined(__AVX512F__) && defined(__AVX512DQ__)
    Vec8d r; _mm512_storeu_pd(r.e, vlmd_tanh(_mm512_loadu_pd(a.e))); return r;
#else
    return vclc_lanewise_d(a, lmd_tanh);
#endif
}
static inline Vec4d atanh(const Vec4d a) { return vclc_lanewise_d(a, lmd_atanh); }
static inline Vec8d atanh(const Vec8d a) {
#if defined(__AVX512F__) && defined(__AVX512DQ__)
    Vec8d r; _mm512_storeu_pd(r.e, vlmd_atanh(_mm512_loadu_pd(a.e))); return r;
#else
    return vclc_lanewise_d(a, lmd_atanh);
#endif
}
#endif
