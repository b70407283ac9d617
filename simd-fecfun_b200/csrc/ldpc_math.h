/* Shared float32 (and float64, below) tanh / atanh for the sum-product decoder.
 *
 * The reference's sum-product check update evaluates tanh(|Q|/2), multiplies
 * the results along a fixed tree, clamps at Max_val and applies 2*atanh
 * (src/LDPCDec/min_find.pl:37-48 and 98-106).  Its tanh/atanh come from the
 * third-party vectorclass header vectormath_hyp.h, which is not part of the
 * reference tree.  Near the clamp (1 - 2^-24) one ulp of the product moves
 * 2*atanh by ~0.7, so the GPU decoder and the CPU oracle must use the *same*
 * function, bit for bit.  This header is that function.  It uses only IEEE
 * single-precision +, -, *, /, fused multiply-add and round-to-nearest-even,
 * each correctly rounded, written so that no compiler may contract or
 * reassociate them:
 *   - device code calls __fmul_rn/__fadd_rn/__fsub_rn/__fdiv_rn/__fmaf_rn;
 *   - host code calls fmaf for the fused steps and must be compiled with
 *     -ffp-contract=off for the others.
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
#define LM_FMA(a, b, c) __fmaf_rn((a), (b), (c))
#else
#include <math.h>
#define LM_MUL(a, b) ((float)(a) * (float)(b))
#define LM_ADD(a, b) ((float)(a) + (float)(b))
#define LM_SUB(a, b) ((float)(a) - (float)(b))
#define LM_DIV(a, b) ((float)(a) / (float)(b))
#define LM_FMA(a, b, c) fmaf((float)(a), (float)(b), (float)(c))
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
    float r = LM_FMA(-k, ln2_lo, LM_FMA(-k, ln2_hi, y));
    /* e^r, |r| <= 0.35, Taylor to r^8 (Horner) */
    float p = 2.4801587301587302e-05f;                 /* 1/8! */
    p = LM_FMA(p, r, 1.9841269841269841e-04f); /* 1/7! */
    p = LM_FMA(p, r, 1.3888888888888889e-03f); /* 1/6! */
    p = LM_FMA(p, r, 8.3333333333333333e-03f); /* 1/5! */
    p = LM_FMA(p, r, 4.1666666666666667e-02f); /* 1/4! */
    p = LM_FMA(p, r, 1.6666666666666667e-01f); /* 1/3! */
    p = LM_FMA(p, r, 0.5f);
    p = LM_FMA(p, r, 1.0f);
    p = LM_FMA(p, r, 1.0f);
    int32_t ki = (int32_t)k;                          /* -44 <= ki <= 0 */
    return LM_MUL(p, lm_i2f((127 + ki) << 23));
}

/* expm1(y) for -30 <= y <= 0, accurate relative to the result near 0 */
LM_FN float lm_expm1_neg(float y) {
    if (y > -0.25f) {
        float p = 2.7557319223985891e-06f;                 /* 1/9! */
        p = LM_FMA(p, y, 2.4801587301587302e-05f); /* 1/8! */
        p = LM_FMA(p, y, 1.9841269841269841e-04f);
        p = LM_FMA(p, y, 1.3888888888888889e-03f);
        p = LM_FMA(p, y, 8.3333333333333333e-03f);
        p = LM_FMA(p, y, 4.1666666666666667e-02f);
        p = LM_FMA(p, y, 1.6666666666666667e-01f);
        p = LM_FMA(p, y, 0.5f);
        p = LM_FMA(p, y, 1.0f);
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
    p = LM_FMA(p, s2, 9.0909090909090909e-02f);
    p = LM_FMA(p, s2, 1.1111111111111111e-01f);
    p = LM_FMA(p, s2, 1.4285714285714286e-01f);
    p = LM_FMA(p, s2, 2.0000000000000000e-01f);
    p = LM_FMA(p, s2, 3.3333333333333333e-01f);
    p = LM_FMA(p, s2, 1.0f);
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
    float lo = LM_ADD(LM_FMA(ef, ln2_lo, lm_log_series(s)), corr);
    return LM_FMA(ef, ln2_hi, lo);
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

/* ---- double precision (the reference's SIMD_ELEM_BW=-64 builds) ----------
 *
 * Same methods as above, carried to double precision: Cody-Waite reduction
 * with ln2 split into a 32-bit head (k*ln2_hi exact for |k| < 2^21) and a
 * tail; e^r Taylor to r^14 (|r| <= 0.347, remainder < 2^-60); expm1 Taylor to
 * y^14 for |y| < 1/4; 2*atanh series to s^25; tanh(x) = 1 for x >= 20
 * (1 - tanh(20) < 2^-57).  The constants are 1/n!, 1/(2k+1), ln2 and 1/ln2
 * rounded to double. */
#if defined(__CUDA_ARCH__)
#define LMD_MUL(a, b) __dmul_rn((a), (b))
#define LMD_ADD(a, b) __dadd_rn((a), (b))
#define LMD_SUB(a, b) __dsub_rn((a), (b))
#define LMD_DIV(a, b) __ddiv_rn((a), (b))
#define LMD_FMA(a, b, c) __fma_rn((a), (b), (c))
#else
#define LMD_MUL(a, b) ((double)(a) * (double)(b))
#define LMD_ADD(a, b) ((double)(a) + (double)(b))
#define LMD_SUB(a, b) ((double)(a) - (double)(b))
#define LMD_DIV(a, b) ((double)(a) / (double)(b))
#define LMD_FMA(a, b, c) fma((double)(a), (double)(b), (double)(c))
#endif

LM_FN int64_t lmd_d2i(double x) {
#if defined(__CUDA_ARCH__)
    return __double_as_longlong(x);
#else
    int64_t i; memcpy(&i, &x, 8); return i;
#endif
}

LM_FN double lmd_i2d(int64_t i) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double(i);
#else
    double x; memcpy(&x, &i, 8); return x;
#endif
}

#define LMD_LN2_HI 0.69314718036912382          /* 32 significant bits */
#define LMD_LN2_LO 1.9082149292705877e-10

/* round to nearest, ties to even, for |x| < 2^51 */
LM_FN double lmd_rint(double x) {
    const double magic = 6755399441055744.0; /* 1.5 * 2^52 */
    return LMD_SUB(LMD_ADD(x, magic), magic);
}

/* e^y for -45 <= y <= 0 */
LM_FN double lmd_exp_neg(double y) {
    const double inv_ln2 = 1.4426950408889634;
    double k = lmd_rint(LMD_MUL(y, inv_ln2));
    double r = LMD_FMA(-k, LMD_LN2_LO, LMD_FMA(-k, LMD_LN2_HI, y));
    double p = 1.1470745597729725e-11;                   /* 1/14! */
    p = LMD_FMA(p, r, 1.6059043836821613e-10); /* 1/13! */
    p = LMD_FMA(p, r, 2.08767569878681e-09);   /* 1/12! */
    p = LMD_FMA(p, r, 2.505210838544172e-08);  /* 1/11! */
    p = LMD_FMA(p, r, 2.7557319223985888e-07); /* 1/10! */
    p = LMD_FMA(p, r, 2.7557319223985893e-06); /* 1/9! */
    p = LMD_FMA(p, r, 2.4801587301587302e-05); /* 1/8! */
    p = LMD_FMA(p, r, 1.9841269841269841e-04); /* 1/7! */
    p = LMD_FMA(p, r, 1.3888888888888889e-03); /* 1/6! */
    p = LMD_FMA(p, r, 8.3333333333333332e-03); /* 1/5! */
    p = LMD_FMA(p, r, 4.1666666666666664e-02); /* 1/4! */
    p = LMD_FMA(p, r, 1.6666666666666666e-01); /* 1/3! */
    p = LMD_FMA(p, r, 0.5);
    p = LMD_FMA(p, r, 1.0);
    p = LMD_FMA(p, r, 1.0);
    int64_t ki = (int64_t)k;                             /* -65 <= ki <= 0 */
    return LMD_MUL(p, lmd_i2d((int64_t)(1023 + ki) << 52));
}

/* expm1(y) for -45 <= y <= 0 */
LM_FN double lmd_expm1_neg(double y) {
    if (y > -0.25) {
        double p = 1.1470745597729725e-11;                   /* 1/14! */
        p = LMD_FMA(p, y, 1.6059043836821613e-10);
        p = LMD_FMA(p, y, 2.08767569878681e-09);
        p = LMD_FMA(p, y, 2.505210838544172e-08);
        p = LMD_FMA(p, y, 2.7557319223985888e-07);
        p = LMD_FMA(p, y, 2.7557319223985893e-06);
        p = LMD_FMA(p, y, 2.4801587301587302e-05);
        p = LMD_FMA(p, y, 1.9841269841269841e-04);
        p = LMD_FMA(p, y, 1.3888888888888889e-03);
        p = LMD_FMA(p, y, 8.3333333333333332e-03);
        p = LMD_FMA(p, y, 4.1666666666666664e-02);
        p = LMD_FMA(p, y, 1.6666666666666666e-01);
        p = LMD_FMA(p, y, 0.5);
        p = LMD_FMA(p, y, 1.0);
        return LMD_MUL(p, y);
    }
    return LMD_SUB(lmd_exp_neg(y), 1.0);
}

/* tanh(x) for x >= 0 */
LM_FN double lmd_tanh_pos(double x) {
    if (!(x < 20.0)) return 1.0;
    double e = lmd_expm1_neg(LMD_MUL(-2.0, x));
    return LMD_DIV(LMD_SUB(0.0, e), LMD_ADD(2.0, e));
}

/* 2 * (s + s^3/3 + ... + s^25/25) */
LM_FN double lmd_log_series(double s) {
    double s2 = LMD_MUL(s, s);
    double p = 0.040000000000000001;                     /* 1/25 */
    p = LMD_FMA(p, s2, 0.043478260869565216);  /* 1/23 */
    p = LMD_FMA(p, s2, 0.047619047619047616);  /* 1/21 */
    p = LMD_FMA(p, s2, 0.052631578947368418);  /* 1/19 */
    p = LMD_FMA(p, s2, 0.058823529411764705);  /* 1/17 */
    p = LMD_FMA(p, s2, 0.066666666666666666);  /* 1/15 */
    p = LMD_FMA(p, s2, 0.076923076923076927);  /* 1/13 */
    p = LMD_FMA(p, s2, 0.090909090909090912);  /* 1/11 */
    p = LMD_FMA(p, s2, 0.1111111111111111);    /* 1/9 */
    p = LMD_FMA(p, s2, 0.14285714285714285);   /* 1/7 */
    p = LMD_FMA(p, s2, 0.20000000000000001);   /* 1/5 */
    p = LMD_FMA(p, s2, 0.33333333333333331);   /* 1/3 */
    p = LMD_FMA(p, s2, 1.0);
    return LMD_MUL(2.0, LMD_MUL(p, s));
}

/* log(1 + t) for t >= 0 */
LM_FN double lmd_log1p_pos(double t) {
    if (t < 0.25) return lmd_log_series(LMD_DIV(t, LMD_ADD(2.0, t)));
    double u = LMD_ADD(1.0, t);
    int64_t iu = lmd_d2i(u);
    int64_t e = ((iu >> 52) & 0x7ff) - 1023;
    double f = lmd_i2d((iu & 0x000fffffffffffffLL) | 0x3ff0000000000000LL); /* [1, 2) */
    if (f > 1.4142135623730951) { f = LMD_MUL(f, 0.5); e += 1; }
    double s = LMD_DIV(LMD_SUB(f, 1.0), LMD_ADD(f, 1.0));
    double ef = (double)e;
    double corr = LMD_DIV(LMD_SUB(t, LMD_SUB(u, 1.0)), u);
    double lo = LMD_ADD(LMD_FMA(ef, LMD_LN2_LO, lmd_log_series(s)), corr);
    return LMD_FMA(ef, LMD_LN2_HI, lo);
}

/* atanh(m) for 0 <= m < 1 */
LM_FN double lmd_atanh_pos(double m) {
    double t = LMD_DIV(LMD_ADD(m, m), LMD_SUB(1.0, m));
    return LMD_MUL(0.5, lmd_log1p_pos(t));
}

LM_FN double lmd_tanh(double x) {
    const int64_t sign = (int64_t)0x8000000000000000ULL;
    double r = lmd_tanh_pos(lmd_i2d(lmd_d2i(x) & ~sign));
    return lmd_i2d(lmd_d2i(r) | (lmd_d2i(x) & sign));
}

LM_FN double lmd_atanh(double m) {
    const int64_t sign = (int64_t)0x8000000000000000ULL;
    double r = lmd_atanh_pos(lmd_i2d(lmd_d2i(m) & ~sign));
    return lmd_i2d(lmd_d2i(r) | (lmd_d2i(m) & sign));
}

#endif /* LDPC_MATH_H */
