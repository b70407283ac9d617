/* Shared float32 tanh / atanh for the sum-product decoder.
 *
 * The reference's sum-product check update evaluates tanh(|Q|/2), multiplies
 * the results along a fixed tree, clamps at Max_val and applies 2*atanh
 * (src/LDPCDec/min_find.pl:37-48 and 98-106).  Its tanh/atanh come from the
 * third-party vectorclass header vectormath_hyp.h, which is not part of the
 * reference tree.  Near the clamp (1 - 2^-24) one ulp of the product moves
 * 2*atanh by ~0.7, so the GPU decoder and the CPU oracle must use the *same*
 * function, bit for bit.  This header is that function.  It uses only IEEE
 * single-precision +, -, *, / and round-to-nearest-even, written so that no
 * compiler may contract them into fused multiply-adds:
 *   - device code calls __fmul_rn/__fadd_rn/__fsub_rn/__fdiv_rn;
 *   - host code must be compiled with -ffp-contract=off.
 *
 * Methods (from the mathematics, not from any library):
 *   expm1(y), y <= 0:  |y| < 1/4: Taylor series to y^9;
 *                      else e^y by Cody-Waite reduction y = k ln2 + r with a
 *                      two-part ln2 and the Taylor series of e^r to r^8.
 *   tanh(x), x >= 0:   -expm1(-2x) / (2 + expm1(-2x)); 1 for x >= 10.
 *   log1p(t), t >= 0:  t < 1/4: 2*atanh-series in s = t/(2+t);
 *                      else u = 1+t = 2^e f, f in [sqrt(1/2), sqrt(2)),
 *                      ln u = e ln2 + 2 atanh((f-1)/(f+1)), plus the
 *                      first-order correction (t - (u-1))/u.
 *   atanh(m), 0<=m<1:  log1p(2m / (1 - m)) / 2.
 */
#ifndef LDPC_MATH_H
#define LDPC_MATH_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define LM_FN __host__ __device__ __forceinline__
#else
#define LM_FN static inline
#endif

#if defined(__CUDA_ARCH__)
#define LM_MUL(a, b) __fmul_rn((a), (b))
#define LM_ADD(a, b) __fadd_rn((a), (b))
#define LM_SUB(a, b) __fsub_rn((a), (b))
#define LM_DIV(a, b) __fdiv_rn((a), (b))
#else
#define LM_MUL(a, b) ((float)(a) * (float)(b))
#define LM_ADD(a, b) ((float)(a) + (float)(b))
#define LM_SUB(a, b) ((float)(a) - (float)(b))
#define LM_DIV(a, b) ((float)(a) / (float)(b))
#endif

LM_FN int32_t lm_f2i(float x) {
#if defined(__CUDA_ARCH__)
    return __float_as_int(x);
#else
    int32_t i; memcpy(&i, &x, 4); return i;
#endif
}

LM_FN float lm_i2f(int32_t i) {
#if defined(__CUDA_ARCH__)
    return __int_as_float(i);
#else
    float x; memcpy(&x, &i, 4); return x;
#endif
}

/* round to nearest, ties to even, for |x| < 2^22 (magic-number method) */
LM_FN float lm_rint(float x) {
    const float magic = 12582912.0f; /* 1.5 * 2^23 */
    return LM_SUB(LM_ADD(x, magic), magic);
}

/* e^y for -30 <= y <= 0 */
LM_FN float lm_exp_neg(float y) {
    const float inv_ln2 = 1.44269502162933349609375f;
    const float ln2_hi = 0.693145751953125f;          /* 12 significant bits: k*ln2_hi exact */
    const float ln2_lo = 1.428606765330187045e-06f;
    float k = lm_rint(LM_MUL(y, inv_ln2));
    float r = LM_SUB(LM_SUB(y, LM_MUL(k, ln2_hi)), LM_MUL(k, ln2_lo));
    /* e^r, |r| <= 0.35, Taylor to r^8 (Horner) */
    float p = 2.4801587301587302e-05f;                 /* 1/8! */
    p = LM_ADD(LM_MUL(p, r), 1.9841269841269841e-04f); /* 1/7! */
    p = LM_ADD(LM_MUL(p, r), 1.3888888888888889e-03f); /* 1/6! */
    p = LM_ADD(LM_MUL(p, r), 8.3333333333333333e-03f); /* 1/5! */
    p = LM_ADD(LM_MUL(p, r), 4.1666666666666667e-02f); /* 1/4! */
    p = LM_ADD(LM_MUL(p, r), 1.6666666666666667e-01f); /* 1/3! */
    p = LM_ADD(LM_MUL(p, r), 0.5f);
    p = LM_ADD(LM_MUL(p, r), 1.0f);
    p = LM_ADD(LM_MUL(p, r), 1.0f);
    int32_t ki = (int32_t)k;                          /* -44 <= ki <= 0 */
    return LM_MUL(p, lm_i2f((127 + ki) << 23));
}

/* expm1(y) for -30 <= y <= 0, accurate relative to the result near 0 */
LM_FN float lm_expm1_neg(float y) {
    if (y > -0.25f) {
        float p = 2.7557319223985891e-06f;                 /* 1/9! */
        p = LM_ADD(LM_MUL(p, y), 2.4801587301587302e-05f); /* 1/8! */
        p = LM_ADD(LM_MUL(p, y), 1.9841269841269841e-04f);
        p = LM_ADD(LM_MUL(p, y), 1.3888888888888889e-03f);
        p = LM_ADD(LM_MUL(p, y), 8.3333333333333333e-03f);
        p = LM_ADD(LM_MUL(p, y), 4.1666666666666667e-02f);
        p = LM_ADD(LM_MUL(p, y), 1.6666666666666667e-01f);
        p = LM_ADD(LM_MUL(p, y), 0.5f);
        p = LM_ADD(LM_MUL(p, y), 1.0f);
        return LM_MUL(p, y);
    }
    return LM_SUB(lm_exp_neg(y), 1.0f);
}

/* tanh(x) for x >= 0 (the decoder only ever passes |Q|/2) */
LM_FN float lm_tanh_pos(float x) {
    if (!(x < 10.0f)) return 1.0f;
    float e = lm_expm1_neg(LM_MUL(-2.0f, x));
    return LM_DIV(LM_SUB(0.0f, e), LM_ADD(2.0f, e));
}

/* 2 * atanh-series: s + s^3/3 + ... + s^13/13, times 2 */
LM_FN float lm_log_series(float s) {
    float s2 = LM_MUL(s, s);
    float p = 7.6923076923076923e-02f;            /* 1/13 */
    p = LM_ADD(LM_MUL(p, s2), 9.0909090909090909e-02f);
    p = LM_ADD(LM_MUL(p, s2), 1.1111111111111111e-01f);
    p = LM_ADD(LM_MUL(p, s2), 1.4285714285714286e-01f);
    p = LM_ADD(LM_MUL(p, s2), 2.0000000000000000e-01f);
    p = LM_ADD(LM_MUL(p, s2), 3.3333333333333333e-01f);
    p = LM_ADD(LM_MUL(p, s2), 1.0f);
    return LM_MUL(2.0f, LM_MUL(p, s));
}

/* log(1 + t) for t >= 0 */
LM_FN float lm_log1p_pos(float t) {
    if (t < 0.25f) {
        return lm_log_series(LM_DIV(t, LM_ADD(2.0f, t)));
    }
    const float ln2_hi = 0.693145751953125f;
    const float ln2_lo = 1.428606765330187045e-06f;
    float u = LM_ADD(1.0f, t);
    int32_t iu = lm_f2i(u);
    int32_t e = ((iu >> 23) & 0xff) - 127;
    float f = lm_i2f((iu & 0x007fffff) | 0x3f800000); /* [1, 2) */
    if (f > 1.41421356f) { f = LM_MUL(f, 0.5f); e += 1; }
    float s = LM_DIV(LM_SUB(f, 1.0f), LM_ADD(f, 1.0f));
    float ef = (float)e;
    float corr = LM_DIV(LM_SUB(t, LM_SUB(u, 1.0f)), u);
    float lo = LM_ADD(LM_ADD(LM_MUL(ef, ln2_lo), lm_log_series(s)), corr);
    return LM_ADD(LM_MUL(ef, ln2_hi), lo);
}

/* atanh(m) for 0 <= m < 1 */
LM_FN float lm_atanh_pos(float m) {
    float t = LM_DIV(LM_ADD(m, m), LM_SUB(1.0f, m));
    return LM_MUL(0.5f, lm_log1p_pos(t));
}

/* signed wrappers (the reference's vectorclass tanh/atanh accept any sign) */
LM_FN float lm_tanh(float x) {
    float a = lm_i2f(lm_f2i(x) & 0x7fffffff);
    float r = lm_tanh_pos(a);
    return lm_i2f(lm_f2i(r) | (lm_f2i(x) & (int32_t)0x80000000));
}

LM_FN float lm_atanh(float m) {
    float a = lm_i2f(lm_f2i(m) & 0x7fffffff);
    float r = lm_atanh_pos(a);
    return lm_i2f(lm_f2i(r) | (lm_f2i(m) & (int32_t)0x80000000));
}

#endif /* LDPC_MATH_H */
