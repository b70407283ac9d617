/* vectorclass.h -- compatibility header for building the reference's own
 * C++ sources in this container (oracle / CPU-baseline only).
 *
 * The reference (tomt-1/simd-fecfun) is written against Agner Fog's
 * "vectorclass" library, version 2 (github.com/vectorclass/version2; the
 * reference pins no release: README.md:3,21, build/Makefile:5-7), which is not
 * present here.  This header provides exactly the subset of that library's
 * public API the reference calls, implemented from the library's documented
 * semantics (manual "VCL version 2"):
 *   - integer + - * wrap around; add_saturated/sub_saturated saturate;
 *   - abs() of the most negative integer returns it unchanged;
 *   - min/max of floats return the second operand when the first compares
 *     false (as _mm_min_ps/_mm_max_ps do);
 *   - roundi() rounds to nearest, ties to even;
 *   - compress() truncates; load_partial() zero-fills; cutoff() zeroes tail;
 *   - permuteN<i...>() with index -1 yields zero;
 *   - mul_add() is a fused multiply-add.
 * Lane-generic C++ with AVX-512BW fast paths for the 64 x int8 operations
 * the decoder's inner loops use, and AVX2 paths for the 32-byte vectors of
 * the noise generator and gen_metrics (each the same wrap-around integer or
 * correctly rounded float operation as the lane loop it replaces).  This is test infrastructure: nothing in
 * the shipped library includes it.
 */
#ifndef VCL_COMPAT_VECTORCLASS_H
#define VCL_COMPAT_VECTORCLASS_H

#include <stdint.h>
#include <string.h>
#include <math.h>
#include <type_traits>
#include <immintrin.h>

namespace vclc {

template <int BYTES> struct Raw {
    unsigned char b[BYTES];
};

/* Boolean vector as a bit mask (lane i = bit i), like AVX-512 mask registers. */
template <int N> struct VecB {
    static_assert(N <= 64, "boolean vectors up to 64 lanes");
    uint64_t bits;
    static constexpr uint64_t all() { return N == 64 ? ~0ull : ((1ull << N) - 1); }
    VecB() = default;
    void load_bits(uint64_t b) { bits = b & all(); }
    bool get(int i) const { return (bits >> i) & 1; }
    friend uint64_t to_bits(const VecB& v) { return v.bits; }
    friend VecB operator&(const VecB& a, const VecB& b) { VecB r; r.bits = a.bits & b.bits; return r; }
    friend VecB operator|(const VecB& a, const VecB& b) { VecB r; r.bits = a.bits | b.bits; return r; }
    friend VecB operator~(const VecB& a) { VecB r; r.bits = ~a.bits & all(); return r; }
};

#if defined(__AVX2__)
/* 256-bit helpers for the 32-byte vectors (Vec8f/Vec8i/Vec4uq ...): the same
 * wrap-around integer and correctly rounded float operations as the lane
 * loops below. */
static inline __m256i vclc_ld(const void* p) { return _mm256_loadu_si256((const __m256i*)p); }
static inline void vclc_st(void* p, __m256i v) { _mm256_storeu_si256((__m256i*)p, v); }
template <int B> static inline __m256i vclc_add(__m256i a, __m256i b) {
    if constexpr (B == 1) return _mm256_add_epi8(a, b);
    else if constexpr (B == 2) return _mm256_add_epi16(a, b);
    else if constexpr (B == 4) return _mm256_add_epi32(a, b);
    else return _mm256_add_epi64(a, b);
}
template <int B> static inline __m256i vclc_sub(__m256i a, __m256i b) {
    if constexpr (B == 1) return _mm256_sub_epi8(a, b);
    else if constexpr (B == 2) return _mm256_sub_epi16(a, b);
    else if constexpr (B == 4) return _mm256_sub_epi32(a, b);
    else return _mm256_sub_epi64(a, b);
}
/* shifts by a count >= 0; counts of the lane width or more give 0 (left,
 * logical right) or the sign (arithmetic right), like the lane loops */
template <int B> static inline __m256i vclc_sll(__m256i a, int s) {
    const __m128i c = _mm_cvtsi32_si128(s);
    if constexpr (B == 2) return _mm256_sll_epi16(a, c);
    else if constexpr (B == 4) return _mm256_sll_epi32(a, c);
    else return _mm256_sll_epi64(a, c);
}
template <int B, bool SIGNED> static inline __m256i vclc_sr(__m256i a, int s) {
    const __m128i c = _mm_cvtsi32_si128(s);
    if constexpr (!SIGNED) {
        if constexpr (B == 2) return _mm256_srl_epi16(a, c);
        else if constexpr (B == 4) return _mm256_srl_epi32(a, c);
        else return _mm256_srl_epi64(a, c);
    } else {
        if constexpr (B == 2) return _mm256_sra_epi16(a, c);
        else if constexpr (B == 4) return _mm256_sra_epi32(a, c);
        else return _mm256_sra_epi64(a, c);   /* AVX-512VL */
    }
}
#endif

#if defined(__AVX512F__)
/* saturating 32-bit add (sub = true: a - b): the wrapped result, replaced by
 * INT32_MIN / INT32_MAX (by the sign of a) where the operation overflowed */
static inline __m512i vclc_sat32(__m512i a, __m512i b, bool sub) {
    const __m512i r = sub ? _mm512_sub_epi32(a, b) : _mm512_add_epi32(a, b);
    /* overflow: add -- a, b same sign and r differs; sub -- a, b differ and r differs from a */
    const __m512i ov = sub ? _mm512_and_si512(_mm512_xor_si512(a, b), _mm512_xor_si512(a, r))
                           : _mm512_andnot_si512(_mm512_xor_si512(a, b), _mm512_xor_si512(a, r));
    const __mmask16 m = _mm512_movepi32_mask(ov);
    const __m512i lim = _mm512_xor_si512(_mm512_srai_epi32(a, 31), _mm512_set1_epi32(0x7fffffff));
    return _mm512_mask_blend_epi32(m, r, lim);
}
#endif

template <class T> struct sat_lim {
    static constexpr long long lo = std::is_signed<T>::value ? -(1LL << (8 * sizeof(T) - 1)) : 0;
    static constexpr long long hi = std::is_signed<T>::value ? (1LL << (8 * sizeof(T) - 1)) - 1
                                                            : (long long)((1ULL << (8 * sizeof(T))) - 1);
};

template <class T, int N>
struct alignas((sizeof(T) * N) >= 64 ? 64 : (sizeof(T) * N)) Vec {
    static constexpr int BYTES = (int)sizeof(T) * N;
    T e[N];

    Vec() = default;
    Vec(T v) {
#if defined(__AVX512BW__)
        if constexpr (std::is_same<T, int8_t>::value && N == 64) { _mm512_storeu_si512(e, _mm512_set1_epi8(v)); return; }
        if constexpr (std::is_same<T, float>::value && N == 16) { _mm512_storeu_ps(e, _mm512_set1_ps(v)); return; }
#endif
        for (int i = 0; i < N; ++i) e[i] = v;
    }
    Vec(const Raw<BYTES>& r) { memcpy(e, r.b, BYTES); }
    template <class U, int M, class = typename std::enable_if<(int)sizeof(U) * M == BYTES && !(std::is_same<U, T>::value && M == N)>::type>
    explicit Vec(const Vec<U, M>& o) { memcpy(e, o.e, BYTES); }
    template <int H = N / 2, class = typename std::enable_if<(H * 2 == N && H >= 1)>::type>
    Vec(const Vec<T, H>& lo, const Vec<T, H>& hi) { memcpy(e, lo.e, BYTES / 2); memcpy(e + H, hi.e, BYTES / 2); }
    template <class... A, class = typename std::enable_if<(sizeof...(A) == N && N > 2)>::type>
    Vec(A... a) { T t[N] = {(T)a...}; memcpy(e, t, BYTES); }

    Vec& load(const void* p) { memcpy(e, p, BYTES); return *this; }
    Vec& load_a(const void* p) { memcpy(e, p, BYTES); return *this; }
    void store(void* p) const { memcpy(p, e, BYTES); }
    void store_a(void* p) const { memcpy(p, e, BYTES); }
    Vec& load_partial(int n, const void* p) {
        if (n < 0) n = 0;
        if (n > N) n = N;
        memset(e, 0, BYTES);
        memcpy(e, p, (size_t)n * sizeof(T));
        return *this;
    }
    void store_partial(int n, void* p) const {
        if (n < 0) n = 0;
        if (n > N) n = N;
        memcpy(p, e, (size_t)n * sizeof(T));
    }
    Vec& cutoff(int n) { for (int i = (n < 0 ? 0 : n); i < N; ++i) e[i] = 0; return *this; }
    Vec& insert(int i, T v) { e[i & (N - 1)] = v; return *this; }
    T extract(int i) const { return e[i & (N - 1)]; }
    T operator[](int i) const { return e[i & (N - 1)]; }
    static constexpr int size() { return N; }

    /* ---- bitwise helpers on the raw bytes ---- */
    template <class F> static Vec bitop(const Vec& a, const Vec& b, F f) {
        Vec r; const unsigned char* pa = (const unsigned char*)a.e; const unsigned char* pb = (const unsigned char*)b.e;
        unsigned char* pr = (unsigned char*)r.e;
        for (int i = 0; i < BYTES; ++i) pr[i] = f(pa[i], pb[i]);
        return r;
    }

    friend Vec operator&(const Vec& a, const Vec& b) {
#if defined(__AVX512F__)
        if constexpr (BYTES == 64) { Vec r; _mm512_storeu_si512(r.e, _mm512_and_si512(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r; }
#endif
#if defined(__AVX2__)
        if constexpr (BYTES == 32) { Vec r; vclc_st(r.e, _mm256_and_si256(vclc_ld(a.e), vclc_ld(b.e))); return r; }
#endif
        return bitop(a, b, [](unsigned char x, unsigned char y) { return (unsigned char)(x & y); });
    }
    friend Vec operator|(const Vec& a, const Vec& b) {
#if defined(__AVX512F__)
        if constexpr (BYTES == 64) { Vec r; _mm512_storeu_si512(r.e, _mm512_or_si512(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r; }
#endif
#if defined(__AVX2__)
        if constexpr (BYTES == 32) { Vec r; vclc_st(r.e, _mm256_or_si256(vclc_ld(a.e), vclc_ld(b.e))); return r; }
#endif
        return bitop(a, b, [](unsigned char x, unsigned char y) { return (unsigned char)(x | y); });
    }
    friend Vec operator^(const Vec& a, const Vec& b) {
#if defined(__AVX512F__)
        if constexpr (BYTES == 64) { Vec r; _mm512_storeu_si512(r.e, _mm512_xor_si512(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r; }
#endif
#if defined(__AVX2__)
        if constexpr (BYTES == 32) { Vec r; vclc_st(r.e, _mm256_xor_si256(vclc_ld(a.e), vclc_ld(b.e))); return r; }
#endif
        return bitop(a, b, [](unsigned char x, unsigned char y) { return (unsigned char)(x ^ y); });
    }
    friend Vec operator~(const Vec& a) {
        Vec r; const unsigned char* pa = (const unsigned char*)a.e; unsigned char* pr = (unsigned char*)r.e;
        for (int i = 0; i < BYTES; ++i) pr[i] = (unsigned char)~pa[i];
        return r;
    }
    friend Vec andnot(const Vec& a, const Vec& b) { return a & ~b; }
    Vec& operator&=(const Vec& b) { *this = *this & b; return *this; }
    Vec& operator|=(const Vec& b) { *this = *this | b; return *this; }
    Vec& operator^=(const Vec& b) { *this = *this ^ b; return *this; }

    /* ---- arithmetic ---- */
    friend Vec operator+(const Vec& a, const Vec& b) {
        Vec r;
#if defined(__AVX512BW__)
        if constexpr (std::is_same<T, int8_t>::value && N == 64) { _mm512_storeu_si512(r.e, _mm512_add_epi8(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r; }
        if constexpr (std::is_same<T, int16_t>::value && N == 32) { _mm512_storeu_si512(r.e, _mm512_add_epi16(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r; }
        if constexpr (std::is_same<T, int32_t>::value && N == 16) { _mm512_storeu_si512(r.e, _mm512_add_epi32(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r; }
        if constexpr (std::is_same<T, float>::value && N == 16) { _mm512_storeu_ps(r.e, _mm512_add_ps(_mm512_loadu_ps(a.e), _mm512_loadu_ps(b.e))); return r; }
#endif
#if defined(__AVX2__)
        if constexpr (BYTES == 32 && std::is_integral<T>::value) { vclc_st(r.e, vclc_add<sizeof(T)>(vclc_ld(a.e), vclc_ld(b.e))); return r; }
        if constexpr (std::is_same<T, float>::value && N == 8) { _mm256_storeu_ps(r.e, _mm256_add_ps(_mm256_loadu_ps(a.e), _mm256_loadu_ps(b.e))); return r; }
#endif
#if defined(__AVX512F__)
        if constexpr (std::is_same<T, double>::value && N == 8) { _mm512_storeu_pd(r.e, _mm512_add_pd(_mm512_loadu_pd(a.e), _mm512_loadu_pd(b.e))); return r; }
#endif
        if constexpr (std::is_integral<T>::value) {
            using U = typename std::make_unsigned<T>::type;
            for (int i = 0; i < N; ++i) r.e[i] = (T)(U)((U)a.e[i] + (U)b.e[i]);
        } else {
            for (int i = 0; i < N; ++i) r.e[i] = a.e[i] + b.e[i];
        }
        return r;
    }
    friend Vec operator-(const Vec& a, const Vec& b) {
        Vec r;
#if defined(__AVX512BW__)
        if constexpr (std::is_same<T, int8_t>::value && N == 64) { _mm512_storeu_si512(r.e, _mm512_sub_epi8(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r; }
        if constexpr (std::is_same<T, int16_t>::value && N == 32) { _mm512_storeu_si512(r.e, _mm512_sub_epi16(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r; }
        if constexpr (std::is_same<T, int32_t>::value && N == 16) { _mm512_storeu_si512(r.e, _mm512_sub_epi32(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r; }
        if constexpr (std::is_same<T, float>::value && N == 16) { _mm512_storeu_ps(r.e, _mm512_sub_ps(_mm512_loadu_ps(a.e), _mm512_loadu_ps(b.e))); return r; }
#endif
#if defined(__AVX2__)
        if constexpr (BYTES == 32 && std::is_integral<T>::value) { vclc_st(r.e, vclc_sub<sizeof(T)>(vclc_ld(a.e), vclc_ld(b.e))); return r; }
        if constexpr (std::is_same<T, float>::value && N == 8) { _mm256_storeu_ps(r.e, _mm256_sub_ps(_mm256_loadu_ps(a.e), _mm256_loadu_ps(b.e))); return r; }
#endif
#if defined(__AVX512F__)
        if constexpr (std::is_same<T, double>::value && N == 8) { _mm512_storeu_pd(r.e, _mm512_sub_pd(_mm512_loadu_pd(a.e), _mm512_loadu_pd(b.e))); return r; }
#endif
        if constexpr (std::is_integral<T>::value) {
            using U = typename std::make_unsigned<T>::type;
            for (int i = 0; i < N; ++i) r.e[i] = (T)(U)((U)a.e[i] - (U)b.e[i]);
        } else {
            for (int i = 0; i < N; ++i) r.e[i] = a.e[i] - b.e[i];
        }
        return r;
    }
    friend Vec operator*(const Vec& a, const Vec& b) {
        Vec r;
#if defined(__AVX2__)
        if constexpr (std::is_same<T, float>::value && N == 8) { _mm256_storeu_ps(r.e, _mm256_mul_ps(_mm256_loadu_ps(a.e), _mm256_loadu_ps(b.e))); return r; }
#endif
#if defined(__AVX512F__)
        if constexpr (std::is_same<T, float>::value && N == 16) { _mm512_storeu_ps(r.e, _mm512_mul_ps(_mm512_loadu_ps(a.e), _mm512_loadu_ps(b.e))); return r; }
        if constexpr (std::is_same<T, double>::value && N == 8) { _mm512_storeu_pd(r.e, _mm512_mul_pd(_mm512_loadu_pd(a.e), _mm512_loadu_pd(b.e))); return r; }
#endif
        if constexpr (std::is_integral<T>::value) {
            using U = typename std::make_unsigned<T>::type;
            for (int i = 0; i < N; ++i) r.e[i] = (T)(U)((U)a.e[i] * (U)b.e[i]);
        } else {
            for (int i = 0; i < N; ++i) r.e[i] = a.e[i] * b.e[i];
        }
        return r;
    }
    friend Vec operator/(const Vec& a, const Vec& b) { Vec r; for (int i = 0; i < N; ++i) r.e[i] = a.e[i] / b.e[i]; return r; }
    friend Vec operator-(const Vec& a) { return Vec((T)0) - a; }
    Vec& operator+=(const Vec& b) { *this = *this + b; return *this; }
    Vec& operator-=(const Vec& b) { *this = *this - b; return *this; }
    Vec& operator*=(const Vec& b) { *this = *this * b; return *this; }

    friend Vec operator<<(const Vec& a, int s) {
#if defined(__AVX2__)
        if constexpr (BYTES == 32 && sizeof(T) >= 2 && std::is_integral<T>::value) {
            if (s >= 0) { Vec r; vclc_st(r.e, vclc_sll<sizeof(T)>(vclc_ld(a.e), s)); return r; }
        }
#endif
        Vec r; using U = typename std::make_unsigned<T>::type;
        for (int i = 0; i < N; ++i) r.e[i] = (s >= (int)(8 * sizeof(T))) ? (T)0 : (T)(U)((U)a.e[i] << s);
        return r;
    }
    friend Vec operator>>(const Vec& a, int s) {
#if defined(__AVX2__)
        if constexpr (BYTES == 32 && sizeof(T) >= 2 && std::is_integral<T>::value) {
            if (s >= 0) { Vec r; vclc_st(r.e, vclc_sr<sizeof(T), std::is_signed<T>::value>(vclc_ld(a.e), s)); return r; }
        }
#endif
        Vec r;
        for (int i = 0; i < N; ++i) {
            if (s >= (int)(8 * sizeof(T))) r.e[i] = std::is_signed<T>::value ? (T)(a.e[i] < 0 ? -1 : 0) : (T)0;
            else r.e[i] = (T)(a.e[i] >> s);   /* arithmetic for signed, logical for unsigned */
        }
        return r;
    }

    /* ---- comparisons ---- */
    template <class F> static VecB<N> cmp(const Vec& a, const Vec& b, F f) {
        VecB<N> r; r.bits = 0;
        for (int i = 0; i < N; ++i) r.bits |= (uint64_t)(f(a.e[i], b.e[i]) ? 1 : 0) << i;
        return r;
    }
#if defined(__AVX512BW__) && defined(__AVX512VL__)
    template <int P> static bool cmp_fast(const Vec& a, const Vec& b, VecB<N>& r) {
        if constexpr (std::is_same<T, int8_t>::value && N == 64) { r.bits = _mm512_cmp_epi8_mask(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e), P); return true; }
        if constexpr (std::is_same<T, int16_t>::value && N == 32) { r.bits = _mm512_cmp_epi16_mask(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e), P); return true; }
        if constexpr (std::is_same<T, int32_t>::value && N == 16) { r.bits = _mm512_cmp_epi32_mask(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e), P); return true; }
        if constexpr (std::is_same<T, int32_t>::value && N == 8) { r.bits = _mm256_cmp_epi32_mask(_mm256_loadu_si256((const __m256i*)a.e), _mm256_loadu_si256((const __m256i*)b.e), P); return true; }
        return false;
    }
#endif
    friend VecB<N> operator<(const Vec& a, const Vec& b) {
#if defined(__AVX512BW__) && defined(__AVX512VL__)
        { VecB<N> r; if (cmp_fast<_MM_CMPINT_LT>(a, b, r)) return r; }
        if constexpr (std::is_same<T, float>::value && N == 16) { VecB<N> r; r.bits = _mm512_cmp_ps_mask(_mm512_loadu_ps(a.e), _mm512_loadu_ps(b.e), _CMP_LT_OQ); return r; }
        if constexpr (std::is_same<T, float>::value && N == 8) { VecB<N> r; r.bits = _mm256_cmp_ps_mask(_mm256_loadu_ps(a.e), _mm256_loadu_ps(b.e), _CMP_LT_OQ); return r; }
#endif
        return cmp(a, b, [](T x, T y) { return x < y; });
    }
    friend VecB<N> operator>(const Vec& a, const Vec& b) { return b < a; }
    friend VecB<N> operator<=(const Vec& a, const Vec& b) { return cmp(a, b, [](T x, T y) { return x <= y; }); }
    friend VecB<N> operator>=(const Vec& a, const Vec& b) { return b <= a; }
    friend VecB<N> operator==(const Vec& a, const Vec& b) {
#if defined(__AVX512BW__) && defined(__AVX512VL__)
        { VecB<N> r; if (cmp_fast<_MM_CMPINT_EQ>(a, b, r)) return r; }
#endif
        return cmp(a, b, [](T x, T y) { return x == y; });
    }
    friend VecB<N> operator!=(const Vec& a, const Vec& b) { return cmp(a, b, [](T x, T y) { return x != y; }); }

    /* ---- element functions ---- */
    friend Vec select(const VecB<N>& s, const Vec& a, const Vec& b) {
#if defined(__AVX512BW__)
        if constexpr (std::is_same<T, int8_t>::value && N == 64) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_mask_blend_epi8((__mmask64)s.bits, _mm512_loadu_si512(b.e), _mm512_loadu_si512(a.e)));
            return r;
        }
#endif
#if defined(__AVX512BW__) && defined(__AVX512VL__)
        if constexpr (BYTES == 64 && sizeof(T) == 2) { Vec r; _mm512_storeu_si512(r.e, _mm512_mask_blend_epi16((__mmask32)s.bits, _mm512_loadu_si512(b.e), _mm512_loadu_si512(a.e))); return r; }
        if constexpr (BYTES == 64 && sizeof(T) == 4) { Vec r; _mm512_storeu_si512(r.e, _mm512_mask_blend_epi32((__mmask16)s.bits, _mm512_loadu_si512(b.e), _mm512_loadu_si512(a.e))); return r; }
        if constexpr (BYTES == 32 && sizeof(T) == 4) { Vec r; _mm256_storeu_si256((__m256i*)r.e, _mm256_mask_blend_epi32((__mmask8)s.bits, _mm256_loadu_si256((const __m256i*)b.e), _mm256_loadu_si256((const __m256i*)a.e))); return r; }
#endif
        Vec r; for (int i = 0; i < N; ++i) r.e[i] = s.get(i) ? a.e[i] : b.e[i]; return r;
    }
    friend Vec if_sub(const VecB<N>& s, const Vec& a, const Vec& b) { return select(s, a - b, a); }
    friend Vec if_add(const VecB<N>& s, const Vec& a, const Vec& b) { return select(s, a + b, a); }
    friend Vec min(const Vec& a, const Vec& b) {
#if defined(__AVX512BW__)
        if constexpr (std::is_same<T, int8_t>::value && N == 64) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_min_epi8(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r;
        }
        if constexpr (std::is_same<T, int16_t>::value && N == 32) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_min_epi16(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r;
        }
        if constexpr (std::is_same<T, int32_t>::value && N == 16) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_min_epi32(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r;
        }
#endif
#if defined(__AVX2__)
        /* minps: the second operand unless the first compares less, as below */
        if constexpr (std::is_same<T, float>::value && N == 8) { Vec r; _mm256_storeu_ps(r.e, _mm256_min_ps(_mm256_loadu_ps(a.e), _mm256_loadu_ps(b.e))); return r; }
#endif
#if defined(__AVX512F__)
        if constexpr (std::is_same<T, float>::value && N == 16) { Vec r; _mm512_storeu_ps(r.e, _mm512_min_ps(_mm512_loadu_ps(a.e), _mm512_loadu_ps(b.e))); return r; }
        if constexpr (std::is_same<T, double>::value && N == 8) { Vec r; _mm512_storeu_pd(r.e, _mm512_min_pd(_mm512_loadu_pd(a.e), _mm512_loadu_pd(b.e))); return r; }
#endif
        Vec r; for (int i = 0; i < N; ++i) r.e[i] = (a.e[i] < b.e[i]) ? a.e[i] : b.e[i]; return r;
    }
    friend Vec max(const Vec& a, const Vec& b) {
#if defined(__AVX512BW__)
        if constexpr (std::is_same<T, int8_t>::value && N == 64) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_max_epi8(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r;
        }
        if constexpr (std::is_same<T, int16_t>::value && N == 32) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_max_epi16(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r;
        }
        if constexpr (std::is_same<T, int32_t>::value && N == 16) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_max_epi32(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r;
        }
#endif
#if defined(__AVX2__)
        if constexpr (std::is_same<T, float>::value && N == 8) { Vec r; _mm256_storeu_ps(r.e, _mm256_max_ps(_mm256_loadu_ps(a.e), _mm256_loadu_ps(b.e))); return r; }
#endif
#if defined(__AVX512F__)
        if constexpr (std::is_same<T, float>::value && N == 16) { Vec r; _mm512_storeu_ps(r.e, _mm512_max_ps(_mm512_loadu_ps(a.e), _mm512_loadu_ps(b.e))); return r; }
        if constexpr (std::is_same<T, double>::value && N == 8) { Vec r; _mm512_storeu_pd(r.e, _mm512_max_pd(_mm512_loadu_pd(a.e), _mm512_loadu_pd(b.e))); return r; }
#endif
        Vec r; for (int i = 0; i < N; ++i) r.e[i] = (a.e[i] > b.e[i]) ? a.e[i] : b.e[i]; return r;
    }
    friend Vec abs(const Vec& a) {
        Vec r;
        if constexpr (std::is_integral<T>::value) {
#if defined(__AVX512BW__)
            if constexpr (std::is_same<T, int8_t>::value && N == 64) {
                _mm512_storeu_si512(r.e, _mm512_abs_epi8(_mm512_loadu_si512(a.e))); return r;
            }
            if constexpr (std::is_same<T, int16_t>::value && N == 32) {
                _mm512_storeu_si512(r.e, _mm512_abs_epi16(_mm512_loadu_si512(a.e))); return r;
            }
            if constexpr (std::is_same<T, int32_t>::value && N == 16) {
                _mm512_storeu_si512(r.e, _mm512_abs_epi32(_mm512_loadu_si512(a.e))); return r;
            }
#endif
            using U = typename std::make_unsigned<T>::type;
            for (int i = 0; i < N; ++i) r.e[i] = (a.e[i] < 0) ? (T)(U)(0u - (U)a.e[i]) : a.e[i];
        } else {
#if defined(__AVX512F__)
            if constexpr (BYTES == 64) {   /* fabs: clear the sign bits */
                const __m512i m = sizeof(T) == 4 ? _mm512_set1_epi32(0x7fffffff) : _mm512_set1_epi64(0x7fffffffffffffffLL);
                _mm512_storeu_si512(r.e, _mm512_and_si512(_mm512_loadu_si512(a.e), m));
                return r;
            }
#endif
            for (int i = 0; i < N; ++i) r.e[i] = fabs(a.e[i]);
        }
        return r;
    }
    friend Vec add_saturated(const Vec& a, const Vec& b) {
#if defined(__AVX512BW__)
        if constexpr (std::is_same<T, int8_t>::value && N == 64) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_adds_epi8(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r;
        }
        if constexpr (std::is_same<T, int16_t>::value && N == 32) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_adds_epi16(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r;
        }
        if constexpr (std::is_same<T, int32_t>::value && N == 16) {
            Vec r; _mm512_storeu_si512(r.e, vclc_sat32(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e), false)); return r;
        }
#endif
        Vec r;
        for (int i = 0; i < N; ++i) {
            long long v = (long long)a.e[i] + (long long)b.e[i];
            r.e[i] = (T)(v < sat_lim<T>::lo ? sat_lim<T>::lo : v > sat_lim<T>::hi ? sat_lim<T>::hi : v);
        }
        return r;
    }
    friend Vec sub_saturated(const Vec& a, const Vec& b) {
#if defined(__AVX512BW__)
        if constexpr (std::is_same<T, int8_t>::value && N == 64) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_subs_epi8(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r;
        }
        if constexpr (std::is_same<T, int16_t>::value && N == 32) {
            Vec r; _mm512_storeu_si512(r.e, _mm512_subs_epi16(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e))); return r;
        }
        if constexpr (std::is_same<T, int32_t>::value && N == 16) {
            Vec r; _mm512_storeu_si512(r.e, vclc_sat32(_mm512_loadu_si512(a.e), _mm512_loadu_si512(b.e), true)); return r;
        }
#endif
        Vec r;
        for (int i = 0; i < N; ++i) {
            long long v = (long long)a.e[i] - (long long)b.e[i];
            r.e[i] = (T)(v < sat_lim<T>::lo ? sat_lim<T>::lo : v > sat_lim<T>::hi ? sat_lim<T>::hi : v);
        }
        return r;
    }
    friend Vec mul_add(const Vec& a, const Vec& b, const Vec& c) {
        Vec r;
#if defined(__AVX2__) && defined(__FMA__)
        if constexpr (std::is_same<T, float>::value && N == 8) {
            _mm256_storeu_ps(r.e, _mm256_fmadd_ps(_mm256_loadu_ps(a.e), _mm256_loadu_ps(b.e), _mm256_loadu_ps(c.e)));
            return r;
        }
#endif
#if defined(__AVX512F__)
        if constexpr (std::is_same<T, float>::value && N == 16) {
            _mm512_storeu_ps(r.e, _mm512_fmadd_ps(_mm512_loadu_ps(a.e), _mm512_loadu_ps(b.e), _mm512_loadu_ps(c.e)));
            return r;
        }
        if constexpr (std::is_same<T, double>::value && N == 8) {
            _mm512_storeu_pd(r.e, _mm512_fmadd_pd(_mm512_loadu_pd(a.e), _mm512_loadu_pd(b.e), _mm512_loadu_pd(c.e)));
            return r;
        }
#endif
        if constexpr (std::is_same<T, float>::value) { for (int i = 0; i < N; ++i) r.e[i] = fmaf(a.e[i], b.e[i], c.e[i]); }
        else if constexpr (std::is_same<T, double>::value) { for (int i = 0; i < N; ++i) r.e[i] = fma(a.e[i], b.e[i], c.e[i]); }
        else { r = a * b + c; }
        return r;
    }
    friend Vec sqrt(const Vec& a) {
        Vec r;
#if defined(__AVX2__)
        if constexpr (std::is_same<T, float>::value && N == 8) { _mm256_storeu_ps(r.e, _mm256_sqrt_ps(_mm256_loadu_ps(a.e))); return r; }
#endif
        if constexpr (std::is_same<T, float>::value) { for (int i = 0; i < N; ++i) r.e[i] = sqrtf(a.e[i]); }
        else { for (int i = 0; i < N; ++i) r.e[i] = (T)::sqrt((double)a.e[i]); }
        return r;
    }
    friend T horizontal_add(const Vec& a) {
        if constexpr (std::is_integral<T>::value) {
            using U = typename std::make_unsigned<T>::type;
            U s = 0; for (int i = 0; i < N; ++i) s = (U)(s + (U)a.e[i]); return (T)s;
        } else {
            T s = 0; for (int i = 0; i < N; ++i) s += a.e[i]; return s;
        }
    }
};

template <class T, int N> Raw<(int)sizeof(T) * N> reinterpret_i(const Vec<T, N>& a) { Raw<(int)sizeof(T) * N> r; memcpy(r.b, a.e, sizeof(r.b)); return r; }
template <class T, int N> Raw<(int)sizeof(T) * N> reinterpret_f(const Vec<T, N>& a) { Raw<(int)sizeof(T) * N> r; memcpy(r.b, a.e, sizeof(r.b)); return r; }
template <int B> Raw<B> reinterpret_i(const Raw<B>& a) { return a; }
template <int B> Raw<B> reinterpret_f(const Raw<B>& a) { return a; }

template <int N> Vec<float, N> to_float(const Vec<int32_t, N>& a) {
    Vec<float, N> r;
#if defined(__AVX2__)
    if constexpr (N == 8) { _mm256_storeu_ps(r.e, _mm256_cvtepi32_ps(vclc_ld(a.e))); return r; }
#endif
    for (int i = 0; i < N; ++i) r.e[i] = (float)a.e[i];
    return r;
}
template <int N> Vec<float, N> to_float(const Vec<uint32_t, N>& a) { Vec<float, N> r; for (int i = 0; i < N; ++i) r.e[i] = (float)a.e[i]; return r; }
template <int N> Vec<double, N> to_double(const Vec<float, N>& a) { Vec<double, N> r; for (int i = 0; i < N; ++i) r.e[i] = (double)a.e[i]; return r; }
template <int N> Vec<int32_t, N> roundi(const Vec<float, N>& a) {
    Vec<int32_t, N> r;
#if defined(__AVX2__)
    /* cvtps2dq rounds by MXCSR (nearest-even by default), as nearbyintf does */
    if constexpr (N == 8) { vclc_st(r.e, _mm256_cvtps_epi32(_mm256_loadu_ps(a.e))); return r; }
#endif
    for (int i = 0; i < N; ++i) r.e[i] = (int32_t)nearbyintf(a.e[i]);
    return r;
}
template <int N> Vec<int32_t, N> truncatei(const Vec<float, N>& a) { Vec<int32_t, N> r; for (int i = 0; i < N; ++i) r.e[i] = (int32_t)a.e[i]; return r; }
template <int N> Vec<int16_t, N> compress(const Vec<int32_t, N>& a) { Vec<int16_t, N> r; for (int i = 0; i < N; ++i) r.e[i] = (int16_t)(uint16_t)(uint32_t)a.e[i]; return r; }

template <class T, int N, int... I> Vec<T, N> permute_impl(const Vec<T, N>& a) {
    static_assert(sizeof...(I) == N, "permute needs one index per element");
    const int idx[N] = {I...};
    Vec<T, N> r;
    for (int i = 0; i < N; ++i) r.e[i] = (idx[i] < 0) ? (T)0 : a.e[idx[i]];
    return r;
}
template <int... I, class T> Vec<T, 4> permute4(const Vec<T, 4>& a) { return permute_impl<T, 4, I...>(a); }
template <int... I, class T> Vec<T, 8> permute8(const Vec<T, 8>& a) { return permute_impl<T, 8, I...>(a); }
template <int... I, class T> Vec<T, 16> permute16(const Vec<T, 16>& a) { return permute_impl<T, 16, I...>(a); }

} /* namespace vclc */

typedef vclc::Vec<int8_t, 16> Vec16c;
typedef vclc::Vec<int8_t, 32> Vec32c;
typedef vclc::Vec<int8_t, 64> Vec64c;
typedef vclc::Vec<int16_t, 8> Vec8s;
typedef vclc::Vec<int16_t, 16> Vec16s;
typedef vclc::Vec<int16_t, 32> Vec32s;
typedef vclc::Vec<int32_t, 4> Vec4i;
typedef vclc::Vec<int32_t, 8> Vec8i;
typedef vclc::Vec<int32_t, 16> Vec16i;
typedef vclc::Vec<uint32_t, 8> Vec8ui;
typedef vclc::Vec<uint32_t, 16> Vec16ui;
typedef vclc::Vec<int64_t, 4> Vec4q;
typedef vclc::Vec<int64_t, 8> Vec8q;
typedef vclc::Vec<uint64_t, 4> Vec4uq;
typedef vclc::Vec<uint64_t, 8> Vec8uq;
typedef vclc::Vec<float, 8> Vec8f;
typedef vclc::Vec<float, 16> Vec16f;
typedef vclc::Vec<double, 4> Vec4d;
typedef vclc::Vec<double, 8> Vec8d;
typedef vclc::VecB<8> Vec8fb;
typedef vclc::VecB<8> Vec8ib;
typedef vclc::VecB<16> Vec16fb;
typedef vclc::VecB<16> Vec16ib;
typedef vclc::VecB<16> Vec16cb;
typedef vclc::VecB<32> Vec32cb;
typedef vclc::VecB<64> Vec64cb;

/* sign_combine(a, b) for float vectors: a with its sign bit flipped where b
 * has the sign bit set (the integer overloads are in the reference's own
 * vectorclass_extensions.h). */
template <class V> static inline V vclc_sign_combine_f(const V& a, const V& b) {
    V r;
#if defined(__AVX512F__)
    if constexpr (V::BYTES == 64) {   /* a with its sign bit flipped where b's is set: a ^ (b & sign) */
        const __m512i m = sizeof(a.e[0]) == 4 ? _mm512_set1_epi32((int)0x80000000u) : _mm512_set1_epi64((long long)0x8000000000000000ULL);
        _mm512_storeu_si512(r.e, _mm512_xor_si512(_mm512_loadu_si512(a.e), _mm512_and_si512(_mm512_loadu_si512(b.e), m)));
        return r;
    }
#endif
    for (int i = 0; i < V::size(); ++i) r.e[i] = std::signbit(b.e[i]) ? -a.e[i] : a.e[i];
    return r;
}
static inline Vec8f sign_combine(const Vec8f a, const Vec8f b) { return vclc_sign_combine_f(a, b); }
static inline Vec16f sign_combine(const Vec16f a, const Vec16f b) { return vclc_sign_combine_f(a, b); }
static inline Vec4d sign_combine(const Vec4d a, const Vec4d b) { return vclc_sign_combine_f(a, b); }
static inline Vec8d sign_combine(const Vec8d a, const Vec8d b) { return vclc_sign_combine_f(a, b); }

using vclc::permute4;
using vclc::permute8;
using vclc::permute16;
using vclc::to_float;
using vclc::to_double;
using vclc::roundi;
using vclc::truncatei;
using vclc::compress;
using vclc::reinterpret_i;
using vclc::reinterpret_f;

#endif /* VCL_COMPAT_VECTORCLASS_H */
