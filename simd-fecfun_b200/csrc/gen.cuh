// Fused channel generation: random data bits -> QC encoding -> BPSK over
// AWGN -> LLR quantisation, for every SNR point, in one kernel.
//
// Reference path replaced (one warp per codeword):
//   gen_rand_databits  src/Top/gen_rand_databits.cpp:11-40   (data bits, filler zeroed)
//   LDPCencode         src/LDPCEnc/LDPCencode.cpp:40-100     (parity column = XOR of
//                      rotated known columns, schedule from LDPCencode.raw.dat)
//   normdist2          src/RNGfunc/prng_functions.cpp:148-186 (Gaussian noise)
//   gen_metrics        src/Top/gen_metrics.cpp:18-121        (BPSK, LLR, clip, puncture,
//                      filler, round-to-nearest-even, int8)
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11), key = seed, counter =
// (codeword lo, codeword hi, block, stream).  Stream 0 gives data bits
// (128 per block), stream 1 gives the noise of bits 4b..4b+3 of block b, and
// stream 2 extends the Gaussian tail.  Gaussians come from the Box-Muller
// transform r = sqrt(-2 ln u1), (r cos 2 pi u2, r sin 2 pi u2) with
// u1 = (w + 1/2) 2^-32; when w < 256 a second word refines u1 down to 2^-65,
// so samples reach ~9.5 sigma (the reference's generator reaches ~9.3 sigma,
// docs/WGN/norm.dist.methods.html).  log2, sqrt and sin/cos are the hardware
// approximations (box_muller_fast); the noise is checked statistically.  The same noise is reused for every SNR
// point, as the reference's inner loop does (src/Top/LDPCtop.cpp:89-97).
#pragma once
#include <stdint.h>

#include "tables.h"

namespace ldpc {

// Term i of the encoder schedule (parameter block, or device memory for
// schedules longer than GEN_MAX_TERMS).
__device__ __forceinline__ int gen_term_col(const GenTables& tb, int i) {
    return tb.term_dev ? tb.term_dev[i] : tb.term_col[i];
}
__device__ __forceinline__ int gen_term_shift(const GenTables& tb, int i) {
    return tb.term_dev ? tb.term_dev[tb.n_terms + i] : tb.term_shift[i];
}

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// The same generator with its ten round keys precomputed (GenJob::philox_rk):
// each key is an operand read from the kernel parameters, not recomputed.
__device__ __forceinline__ uint4 philox_rk(uint64_t cw, uint32_t block, uint32_t stream, const uint32_t (&rk)[20]) {
    uint4 c = make_uint4((uint32_t)cw, (uint32_t)(cw >> 32), block, stream);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ rk[2 * r], lo1, hi0 ^ c.w ^ rk[2 * r + 1], lo0);
    }
    return c;
}

__device__ __forceinline__ uint4 philox_at(uint64_t seed, uint64_t cw, uint32_t block, uint32_t stream) {
    return philox4x32_10(make_uint4((uint32_t)cw, (uint32_t)(cw >> 32), block, stream),
                         make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
}

// gen_metrics for one element: returns 1 for an uncoded sign error.
__device__ __forceinline__ int llr_element(int bit, float noise, float sigma, float sf, float max_abs, int punct,
                                           int filler, float* llr) {
    const float orig = bit ? -1.0f : 1.0f;
    const float rx = fmaf(noise, sigma, orig);
    const int err = (int)((__float_as_uint(orig) ^ __float_as_uint(rx)) >> 31);
    float l = __fmul_rn(rx, sf);
    l = max_abs < l ? max_abs : l;
    l = -max_abs > l ? -max_abs : l;
    if (punct) l = 0.0f;
    if (filler) l = max_abs;
    *llr = l;
    return err;
}

__device__ __forceinline__ int8_t llr_to_i8(float l) {
    return (int8_t)(int16_t)__float2int_rn(l);   // roundi (nearest-even), then compress + byte permute
}

// 32 bits of a z-bit column stored in words[] (one spare zero word after the
// last), starting at bit p (0 <= p < z), wrapping around the column once.
__device__ __forceinline__ uint32_t col_bits32(const uint32_t* words, int z, int p) {
    const int w = p >> 5, sh = p & 31;
    uint32_t v = __funnelshift_r(words[w], words[w + 1], sh);
    const int avail = z - p;
    if (avail < 32) v = (v & ((1u << avail) - 1u)) | (words[0] << avail);
    return v;
}

// 32 bits of a packed bit stream starting at bit p (no wrap).
__device__ __forceinline__ uint32_t stream_bits32(const uint32_t* words, int p) {
    const int w = p >> 5, sh = p & 31;
    return __funnelshift_r(words[w], words[w + 1], sh);
}

// Per-warp shared-memory layout (words):
//   data  [kbits/32 + 2]             data bit stream (filler cleared)
//   cols  [mcol][zw + 1]             columns, zw = ceil(z/32) words each
//   cwbits[n/32 + 2]                 whole codeword as a bit stream
__host__ __device__ inline int gen_warp_words(int kbits, int mcol, int z, int n) {
    const int zw = (z + 31) / 32;
    return (kbits / 32 + 2) + mcol * (zw + 1) + (n / 32 + 2);
}

// Encodes one codeword into the warp's shared memory; data[] must hold the data bits.
__device__ void encode_warp(const GenTables& tb, uint32_t* data, uint32_t* cols, uint32_t* cwbits, int lane) {
    const int z = tb.z, zw = (z + 31) / 32, kc = tb.mcol - tb.mrow;
    const uint32_t last_mask = (z & 31) ? ((1u << (z & 31)) - 1u) : 0xffffffffu;
    // data columns
    for (int i = lane; i < kc * zw; i += 32) {
        const int c = i / zw, k = i - c * zw;
        uint32_t v = stream_bits32(data, c * z + 32 * k);
        if (k == zw - 1) v &= last_mask;
        cols[c * (zw + 1) + k] = v;
    }
    for (int c = lane; c < tb.mcol; c += 32) cols[c * (zw + 1) + zw] = 0u;
    __syncwarp();
    // parity columns in schedule order
    for (int r = 0; r < tb.n_par; ++r) {
        const int pc = tb.par_col[r], first = tb.par_first[r], cnt = tb.par_cnt[r];
        for (int k = lane; k < zw; k += 32) {
            uint32_t acc = 0;
            for (int q = 0; q < cnt; ++q) {
                const int col = gen_term_col(tb, first + q);
                int p = 32 * k + gen_term_shift(tb, first + q);
                p = p % z;
                acc ^= col_bits32(cols + col * (zw + 1), z, p);
            }
            if (k == zw - 1) acc &= last_mask;
            cols[pc * (zw + 1) + k] = acc;
        }
        __syncwarp();
    }
    // concatenate into the codeword bit stream
    const int nw = tb.n / 32 + 2;
    for (int i = lane; i < nw; i += 32) cwbits[i] = 0u;
    __syncwarp();
    for (int i = lane; i < tb.mcol * zw; i += 32) {
        const int c = i / zw, k = i - c * zw;
        const uint32_t v = cols[c * (zw + 1) + k];
        const int o = c * z + 32 * k;
        atomicOr(&cwbits[o >> 5], v << (o & 31));
        if (o & 31) atomicOr(&cwbits[(o >> 5) + 1], v >> (32 - (o & 31)));
    }
    __syncwarp();
}

// Data bits of codeword cw into data[] (kbits bits, filler positions cleared).
__device__ void draw_data_warp(const GenTables& tb, uint64_t seed, uint64_t cw, uint32_t* data, int lane) {
    const int dw = tb.kbits / 32 + 2;
    for (int b = lane; b * 4 < dw; b += 32) {
        const uint4 x = philox_at(seed, cw, (uint32_t)b, 0u);
        const uint32_t v[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int w = 4 * b + q;
            if (w < dw) {
                uint32_t m = v[q];
                const int lo = w * 32;
                if (lo + 32 > tb.kbits) m &= (lo >= tb.kbits) ? 0u : ((1u << (tb.kbits - lo)) - 1u);
                data[w] = m;
            }
        }
    }
    __syncwarp();
    if (tb.any_filler) {
        for (int i = lane; i < tb.kbits; i += 32)
            if (tb.filler[i]) atomicAnd(&data[i >> 5], ~(1u << (i & 31)));
        __syncwarp();
    }
}

// ---- fused generation over tiles of codewords ----
//
// A CTA takes tiles of T consecutive codewords.  Phase A encodes the tile
// into shared memory as bit streams, bits[w * T + c] = word w of codeword c;
// phase B runs the noise and the LLRs of the tile's n/4 four-bit blocks per
// codeword with every thread busy: item f = (c, b) gives one Philox block,
// two Box-Muller pairs and four LLRs per SNR point, stored as one 4-byte word
// per SNR row, so a warp writes 128 contiguous bytes.
//
// Phase A for Z <= 64 and no filler bits (gen_encode_thread): one thread per
// codeword, each column one 64-bit word in shared memory (cols[c * T + t]),
// a parity column the XOR of columns rotated by their shifts.  Otherwise one
// warp per codeword (encode_warp).

constexpr int GEN_THREADS = 256;

// x rotated so that bit i of the result is bit (i + s) mod z of x (z <= 64, s < z)
__device__ __forceinline__ uint64_t rotr_z(uint64_t x, int s, int z, uint64_t mask) {
    return s == 0 ? x : (((x >> s) | (x << (z - s))) & mask);
}

// Per-thread encoder: data words dat[w * T + t] (kbits bits, LSB first) ->
// codeword bit stream bits[w * T + t] (nw words).  cols is 8-byte aligned.
__device__ void gen_encode_thread(const GenTables& tb, const uint32_t* dat, uint64_t* cols, uint32_t* bits, int T,
                                  int t, int nw) {
    const int z = tb.z, kc = tb.mcol - tb.mrow;
    const uint64_t mask = z == 64 ? ~0ull : ((1ull << z) - 1ull);
    for (int c = 0; c < kc; ++c) {
        const int p = c * z, w = p >> 5, sh = p & 31;
        const uint32_t a = dat[w * T + t], b = dat[(w + 1) * T + t], d = dat[(w + 2) * T + t];
        const uint64_t v = (uint64_t)__funnelshift_r(a, b, sh) | ((uint64_t)__funnelshift_r(b, d, sh) << 32);
        cols[c * T + t] = v & mask;
    }
    for (int r = 0; r < tb.n_par; ++r) {
        const int first = tb.par_first[r], cnt = tb.par_cnt[r];
        uint64_t acc = 0;
        for (int q = 0; q < cnt; ++q)
            acc ^= rotr_z(cols[gen_term_col(tb, first + q) * T + t], gen_term_shift(tb, first + q) % z, z, mask);
        cols[tb.par_col[r] * T + t] = acc;
    }
    for (int w = 0; w < nw; ++w) bits[w * T + t] = 0u;
    for (int c = 0; c < tb.mcol; ++c) {
        const uint64_t v = cols[c * T + t];
        const int p = c * z, w = p >> 5, sh = p & 31;
        const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
        bits[w * T + t] |= lo << sh;
        bits[(w + 1) * T + t] |= (sh ? (lo >> (32 - sh)) : 0u) | (hi << sh);
        if (sh) bits[(w + 2) * T + t] |= hi >> (32 - sh);
    }
}

// Box-Muller pair with the hardware approximations of log2, sqrt and
// sin/cos (absolute errors ~2^-21; the noise is checked statistically).
// u1 = (w_r + 1/2) 2^-32, refined by a second word down to 2^-65 when
// w_r < 256 (tail to ~9.5 sigma); angle = pi * (int)w_a * 2^-31 in [-pi, pi).
__device__ __forceinline__ float2 box_muller_fast(uint32_t w_r, uint32_t w_a, const uint32_t (&rk)[20], uint64_t cw,
                                                  uint32_t block, int which) {
    float u1;
    if (w_r < 256u) {
        const uint4 x = philox_rk(cw, block, 2u, rk);
        const uint32_t w2 = which ? x.z : x.x;
        u1 = fmaf((float)w_r, 0x1p-32f, fmaf((float)w2, 0x1p-64f, 0x1p-65f));
    } else {
        u1 = fmaf((float)w_r, 0x1p-32f, 0x1p-33f);
    }
    float r;
    const float e = fmaxf(-1.38629436f * __log2f(u1), 0.0f);   // -2 ln u1 = -2 ln2 log2 u1
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(e));
    float sn, cs;
    __sincosf((float)(int)w_a * 1.46291808e-9f, &sn, &cs);    // pi / 2^31
    return make_float2(r * cs, r * sn);
}

// Sign bit of each of four floats replicated over one byte: byte q = 0xff
// when x_q is negative.
__device__ __forceinline__ uint32_t sign_bytes4(float x0, float x1, float x2, float x3) {
    uint32_t a, b, d;
    asm("prmt.b32 %0, %1, %2, 0x00FB;" : "=r"(a) : "r"(__float_as_uint(x0)), "r"(__float_as_uint(x1)));
    asm("prmt.b32 %0, %1, %2, 0x00FB;" : "=r"(b) : "r"(__float_as_uint(x2)), "r"(__float_as_uint(x3)));
    asm("prmt.b32 %0, %1, %2, 0x5410;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

// Layout of a tile in dynamic shared memory, as the host sizes it:
//   thread encoder (Z <= 64): cols [mcol][T] uint64, dat [dwp][T], bits [nw][T]
//   warp encoder:             bits [nw][T], then per warp gen_warp_words scratch
// with nw = n/32 + 3 and dwp = kbits/32 + 3 (one spare zero word past each
// stream for the encoder's three-word reads and writes).
struct GenTile {
    int T;              // codewords per tile
    int thread_enc;     // 1: gen_encode_thread, 0: encode_warp
    int fast;           // 1: int8 output only, n % 4 == 0, |max_abs| < 2^15, at most GEN_FAST_SNR points
    int clamp16;        // fast path: |rx * sf| < 2^15 at every SNR point, clamp on 16-bit pairs after rounding
    int qshift;         // fast path: items of 4 << qshift elements (n a multiple, int8 output aligned to min(16, item))
};
constexpr int GEN_FAST_SNR = 8;
// fast-path items of up to 16 elements (32 spill registers at 4 CTAs per SM: 3.19 against 2.14 ms)
constexpr int GEN_MAX_QSHIFT = 2;

// gen_metrics for NQ = 4, 8 or 16 consecutive elements at every SNR point,
// the int8 output only:
// rx = fma(noise, sigma, orig) and l = rx * sf as llr_element computes them,
// then the clamp to [-max_abs, max_abs] and roundi: adding 1.5 * 2^23 rounds
// half-even exactly for |l| < 2^21 and leaves roundi(l) in the low bits.
// With clamp16 (the host has bounded |l| < 2^15 at every SNR point) the clamp
// runs after the rounding, on 16-bit lane pairs against +-roundi(max_abs)
// (roundi is monotone, so clamp-then-round equals round-then-clamp to the
// rounded bounds); otherwise it runs on the floats, as llr_element does.
// The low byte of each lane is (int8)(int16)roundi(l).  Punctured elements
// give 0, filler elements roundi(max_abs).  The uncoded error of an element
// is the sign of rx against the sent sign; counts go to unc[s] as four byte
// counters (byte q counts elements q, q + 4, ...), which the kernel folds at
// the end of every tile (the host bounds a thread's items per tile so that no
// byte reaches 256).
__device__ __forceinline__ uint32_t vmax_s16x2(uint32_t a, uint32_t b) { uint32_t d; asm("max.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); return d; }
__device__ __forceinline__ uint32_t vmin_s16x2(uint32_t a, uint32_t b) { uint32_t d; asm("min.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); return d; }

template <int NQ>
__device__ __forceinline__ void llr_i8_fast(const GenJob& job, int8_t* dst, bool clamp16, const float (&nz)[NQ],
                                            uint32_t bitsq, const uint32_t (&pmask)[NQ / 4],
                                            const uint32_t (&fmask)[NQ / 4], uint32_t fbytes, uint32_t lo2, uint32_t hi2,
                                            unsigned (&unc)[GEN_FAST_SNR]) {
    constexpr int W = NQ / 4;   // 32-bit output words per SNR point
    float o[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) o[q] = ((bitsq >> q) & 1u) ? -1.0f : 1.0f;
    uint32_t osign[W];
#pragma unroll
    for (int w = 0; w < W; ++w) osign[w] = sign_bytes4(o[4 * w], o[4 * w + 1], o[4 * w + 2], o[4 * w + 3]);
    const float ma = job.max_abs;
#pragma unroll
    for (int s = 0; s < GEN_FAST_SNR; ++s) {
        if (s < job.n_snr) {
            const float sg = job.sigma[s], sf = job.sigma_factor[s];
            uint32_t packed[W];
            unsigned e = 0;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                // four elements at a time (fewer live registers at 16 per item)
                float rx[4];
                uint32_t t[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    rx[q] = fmaf(nz[4 * w + q], sg, o[4 * w + q]);
                    float l = __fmul_rn(rx[q], sf);
                    if (!clamp16) {
                        l = ma < l ? ma : l;
                        l = -ma > l ? -ma : l;
                    }
                    t[q] = __float_as_uint(__fadd_rn(l, 12582912.0f));
                }
                if (clamp16) {
                    const uint32_t p01 = vmin_s16x2(vmax_s16x2(__byte_perm(t[0], t[1], 0x5410), lo2), hi2);
                    const uint32_t p23 = vmin_s16x2(vmax_s16x2(__byte_perm(t[2], t[3], 0x5410), lo2), hi2);
                    packed[w] = __byte_perm(p01, p23, 0x6420);
                } else {
                    packed[w] = __byte_perm(__byte_perm(t[0], t[1], 0x0040), __byte_perm(t[2], t[3], 0x0040), 0x5410);
                }
                if (pmask[w] | fmask[w]) packed[w] = (packed[w] & ~(pmask[w] | fmask[w])) | (fbytes & fmask[w]);
                e += (sign_bytes4(rx[0], rx[1], rx[2], rx[3]) ^ osign[w]) & 0x01010101u;
            }
            if (W == 1) {
                *reinterpret_cast<uint32_t*>(dst) = packed[0];
            } else if (W == 2) {
                *reinterpret_cast<uint2*>(dst) = make_uint2(packed[0], packed[W - 1]);
            } else {
#pragma unroll
                for (int v = 0; v < W / 4; ++v)
                    *reinterpret_cast<uint4*>(dst + 16 * v) =
                        make_uint4(packed[4 * v], packed[4 * v + 1], packed[4 * v + 2], packed[4 * v + 3]);
            }
            dst += job.snr_stride;
            unc[s] += e;
        }
    }
}

// Phase B of the int8 fast path: item f = codeword c, NQ consecutive bits
// from bit NQ b (n % NQ == 0), one Philox block (counter (cw, block, 1)) and
// two Box-Muller pairs per 4 bits, so every NQ draws the same noise and only
// the per-item work (indices, bit fetch, addresses, one store of NQ bytes per
// SNR point) is shared by NQ elements.  Measured on 802.11ad 1/2 (5 SNR
// points): NQ = 4 2.81 ms, 8 2.38 ms, 16 2.14 ms.
template <int NQ, bool PF>
__device__ __forceinline__ void gen_items_fast(const GenTables& tb, const GenJob& job, const uint32_t* bits, int T,
                                               long long i0, int tc, int tid, bool clamp16,
                                               unsigned (&unc)[GEN_FAST_SNR]) {
    const int nbq = tb.n / NQ;
    const int m = __float2int_rn(job.max_abs);
    const uint32_t hi2 = ((uint32_t)m & 0xffffu) * 0x10001u, lo2 = ((uint32_t)(-m) & 0xffffu) * 0x10001u;
    const uint32_t fbytes = ((uint32_t)m & 0xffu) * 0x01010101u;
    // (c, b) of item f advanced by GEN_THREADS items per step, without a division per item
    int c = tid / nbq, b = tid - (tid / nbq) * nbq;
    const int step_c = GEN_THREADS / nbq, step_b = GEN_THREADS - step_c * nbq;
    for (int f = tid; f < tc * nbq; f += GEN_THREADS, c += step_c, b += step_b) {
        if (b >= nbq) {
            b -= nbq;
            ++c;
        }
        const long long i = i0 + c;
        const uint64_t cw = job.cw_offset + (uint64_t)i;
        const int idx0 = NQ * b;
        float nz[NQ];
#pragma unroll
        for (int h = 0; h < NQ / 4; ++h) {
            const uint32_t blk = (uint32_t)(idx0 / 4 + h);
            const uint4 x = philox_rk(cw, blk, 1u, job.philox_rk);
            const float2 g0 = box_muller_fast(x.x, x.y, job.philox_rk, cw, blk, 0);
            const float2 g1 = box_muller_fast(x.z, x.w, job.philox_rk, cw, blk, 1);
            nz[4 * h] = g0.x;
            nz[4 * h + 1] = g0.y;
            nz[4 * h + 2] = g1.x;
            nz[4 * h + 3] = g1.y;
        }
        const uint32_t bitsq = (bits[(idx0 >> 5) * T + c] >> (idx0 & 31)) & ((1u << NQ) - 1u);
        uint32_t pmask[NQ / 4], fmask[NQ / 4];
#pragma unroll
        for (int w = 0; w < NQ / 4; ++w) {
            pmask[w] = (PF && tb.any_punct) ? *reinterpret_cast<const uint32_t*>(tb.punct + idx0 + 4 * w) * 0xffu : 0u;
            fmask[w] = (PF && tb.any_filler) ? *reinterpret_cast<const uint32_t*>(tb.filler + idx0 + 4 * w) * 0xffu : 0u;
        }
        llr_i8_fast<NQ>(job, job.llr_i8 + i * (long long)tb.n + idx0, clamp16, nz, bitsq, pmask, fmask, fbytes, lo2, hi2,
                        unc);
    }
}

// PF: the code has punctured or filler bits (their masks are applied in the
// int8 path only then).
template <bool PF>
__global__ void __launch_bounds__(GEN_THREADS, 4) gen_kernel(const __grid_constant__ GenTables tb,
                                                          const __grid_constant__ GenJob job, const GenTile tile) {
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ unsigned long long s_unc[GEN_MAX_SNR];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int T = tile.T;
    const int nw = tb.n / 32 + 3, dwp = tb.kbits / 32 + 3, nb = (tb.n + 3) / 4;
    uint64_t* cols = reinterpret_cast<uint64_t*>(sm);
    uint32_t* dat = sm + 2 * tb.mcol * T;
    uint32_t* bits = tile.thread_enc ? dat + dwp * T : sm;
    uint32_t* wscr = sm + nw * T + warp * gen_warp_words(tb.kbits, tb.mcol, tb.z, tb.n);
    for (int i = tid; i < GEN_MAX_SNR; i += blockDim.x) s_unc[i] = 0;
    unsigned unc_f[GEN_FAST_SNR];
#pragma unroll
    for (int s = 0; s < GEN_FAST_SNR; ++s) unc_f[s] = 0;
    const long long ntiles = (job.n_per_snr + T - 1) / T;
    for (long long tl = blockIdx.x; tl < ntiles; tl += gridDim.x) {
        const long long i0 = tl * T;
        const int tc = (int)min((long long)T, job.n_per_snr - i0);
        __syncthreads();   // the previous tile's bits are consumed
        // ---- phase A: data bits and encoding of the tile's codewords ----
        if (tile.thread_enc) {
            if (tid < tc) {
                const uint64_t cw = job.cw_offset + (uint64_t)(i0 + tid);
                for (int b = 0; 4 * b < dwp; ++b) {
                    const uint4 x = philox_rk(cw, (uint32_t)b, 0u, job.philox_rk);
                    const uint32_t v[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int w = 4 * b + q;
                        if (w < dwp) {
                            uint32_t m = v[q];
                            const int lo = w * 32;
                            if (lo + 32 > tb.kbits) m &= (lo >= tb.kbits) ? 0u : ((1u << (tb.kbits - lo)) - 1u);
                            dat[w * T + tid] = m;
                            if (job.data_bits && w < tb.hard_words) job.data_bits[(i0 + tid) * tb.hard_words + w] = m;
                        }
                    }
                }
                gen_encode_thread(tb, dat, cols, bits, T, tid, nw);
            }
        } else {
            uint32_t* data = wscr;
            uint32_t* wcols = data + (tb.kbits / 32 + 2);
            uint32_t* cwbits = wcols + tb.mcol * ((tb.z + 31) / 32 + 1);
            for (int c = warp; c < tc; c += GEN_THREADS / 32) {
                const uint64_t cw = job.cw_offset + (uint64_t)(i0 + c);
                draw_data_warp(tb, job.seed, cw, data, lane);
                if (job.data_bits)
                    for (int w = lane; w < tb.hard_words; w += 32) job.data_bits[(i0 + c) * tb.hard_words + w] = data[w];
                encode_warp(tb, data, wcols, cwbits, lane);
                for (int w = lane; w < tb.n / 32 + 2; w += 32) bits[w * T + c] = cwbits[w];
                __syncwarp();
            }
        }
        __syncthreads();
        // ---- phase B: noise and LLRs, item f = codeword c, block b of 4 bits ----
        if (tile.fast) {
            switch (tile.qshift) {
            case 2: gen_items_fast<16, PF>(tb, job, bits, T, i0, tc, tid, tile.clamp16, unc_f); break;
            case 1: gen_items_fast<8, PF>(tb, job, bits, T, i0, tc, tid, tile.clamp16, unc_f); break;
            default: gen_items_fast<4, PF>(tb, job, bits, T, i0, tc, tid, tile.clamp16, unc_f);
            }
        } else {
            // (c, b) of item f advanced by GEN_THREADS items per step, without a division per item
            int c = tid / nb, b = tid - (tid / nb) * nb;
            const int step_c = GEN_THREADS / nb, step_b = GEN_THREADS - step_c * nb;
            for (int f = tid; f < tc * nb; f += GEN_THREADS, c += step_c, b += step_b) {
                if (b >= nb) {
                    b -= nb;
                    ++c;
                }
                const long long i = i0 + c;
                const uint64_t cw = job.cw_offset + (uint64_t)i;
                const uint4 x = philox_rk(cw, (uint32_t)b, 1u, job.philox_rk);
                const float2 g0 = box_muller_fast(x.x, x.y, job.philox_rk, cw, (uint32_t)b, 0);
                const float2 g1 = box_muller_fast(x.z, x.w, job.philox_rk, cw, (uint32_t)b, 1);
                const float nz[4] = {g0.x, g0.y, g1.x, g1.y};
                const int idx0 = 4 * b;
                const uint32_t bits4 = (bits[(idx0 >> 5) * T + c] >> (idx0 & 31)) & 0xfu;
                for (int s = 0; s < job.n_snr; ++s) {
                    float l[4];
                    uint32_t packed = 0;
                    unsigned e = 0;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int idx = idx0 + q;
                        if (idx < tb.n) {
                            const int pn = tb.any_punct ? tb.punct[idx] : 0;
                            const int fl = tb.any_filler ? tb.filler[idx] : 0;
                            e += llr_element((bits4 >> q) & 1u, nz[q], job.sigma[s], job.sigma_factor[s], job.max_abs, pn,
                                             fl, &l[q]);
                            packed |= (uint32_t)(uint8_t)llr_to_i8(l[q]) << (8 * q);
                        }
                    }
                    if (e && job.uncoded) atomicAdd(&s_unc[s], (unsigned long long)e);
                    const long long row = (long long)s * job.n_per_snr + i;
                    if (job.llr_i8) {
                        int8_t* dst = job.llr_i8 + row * tb.n + idx0;
                        if ((tb.n & 3) == 0) {
                            *reinterpret_cast<uint32_t*>(dst) = packed;
                        } else {
                            for (int q = 0; q < 4 && idx0 + q < tb.n; ++q) dst[q] = (int8_t)(packed >> (8 * q));
                        }
                    }
                    if (job.llr_i16 || job.llr_i32) {
                        for (int q = 0; q < 4 && idx0 + q < tb.n; ++q) {
                            const int v = __float2int_rn(l[q]);           // roundi (nearest-even)
                            if (job.llr_i16) job.llr_i16[row * tb.n + idx0 + q] = (int16_t)v;   // compress: wrap to 16 bits
                            if (job.llr_i32) job.llr_i32[row * tb.n + idx0 + q] = v;
                        }
                    }
                    if (job.llr_f64) {
                        for (int q = 0; q < 4 && idx0 + q < tb.n; ++q) job.llr_f64[row * tb.n + idx0 + q] = (double)l[q];
                    }
                    if (job.llr_f32) {
                        float* dst = job.llr_f32 + row * tb.n + idx0;
                        if ((tb.n & 3) == 0) {
                            *reinterpret_cast<float4*>(dst) = make_float4(l[0], l[1], l[2], l[3]);
                        } else {
                            for (int q = 0; q < 4 && idx0 + q < tb.n; ++q) dst[q] = l[q];
                        }
                    }
                }
            }
        }
        if (tile.fast && job.uncoded) {
            // fold the byte counters of this tile (each byte < 256)
#pragma unroll
            for (int s = 0; s < GEN_FAST_SNR; ++s) {
                if (s < job.n_snr) {
                    const unsigned v = __dp4a(unc_f[s], 0x01010101u, 0u);
                    if (v) atomicAdd(&s_unc[s], (unsigned long long)v);
                    unc_f[s] = 0;
                }
            }
        }
    }
    if (job.uncoded) {
        __syncthreads();
        for (int s = tid; s < job.n_snr; s += blockDim.x)
            if (s_unc[s]) atomicAdd(job.uncoded + s, s_unc[s]);
    }
}

// QC encoding only: packed data bits -> 0/1 codeword bytes.
__global__ void __launch_bounds__(256) encode_kernel(const __grid_constant__ GenTables tb, const uint32_t* data_bits,
                                                     long long n, uint8_t* cw_out) {
    extern __shared__ uint32_t sm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpw = gen_warp_words(tb.kbits, tb.mcol, tb.z, tb.n);
    uint32_t* data = sm + warp * wpw;
    uint32_t* cols = data + (tb.kbits / 32 + 2);
    uint32_t* cwbits = cols + tb.mcol * ((tb.z + 31) / 32 + 1);
    const long long nwarps_total = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long i = (long long)blockIdx.x * (blockDim.x >> 5) + warp; i < n; i += nwarps_total) {
        const int dw = tb.kbits / 32 + 2;
        for (int w = lane; w < dw; w += 32) {
            uint32_t v = w < tb.hard_words ? data_bits[i * tb.hard_words + w] : 0u;
            const int lo = w * 32;
            if (lo + 32 > tb.kbits) v &= (lo >= tb.kbits) ? 0u : ((1u << (tb.kbits - lo)) - 1u);
            data[w] = v;
        }
        __syncwarp();
        encode_warp(tb, data, cols, cwbits, lane);
        for (int idx = lane; idx < tb.n; idx += 32) cw_out[i * tb.n + idx] = (cwbits[idx >> 5] >> (idx & 31)) & 1u;
        __syncwarp();
    }
}

// gen_metrics on given noise: elementwise.
__global__ void llr_from_noise_kernel(const GenTables tb, const uint8_t* bits, const float* noise, long long total,
                                      float sigma, float sf, float max_abs, void* out_int, int int_bytes, float* out_f32,
                                      unsigned long long* uncoded) {
    unsigned long long err = 0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int idx = (int)(e % tb.n);
        float l;
        err += llr_element(bits[e] & 1, noise[e], sigma, sf, max_abs, tb.any_punct ? tb.punct[idx] : 0,
                           tb.any_filler ? tb.filler[idx] : 0, &l);
        if (out_int) {
            if (int_bytes == 1) static_cast<int8_t*>(out_int)[e] = llr_to_i8(l);
            else if (int_bytes == 2) static_cast<int16_t*>(out_int)[e] = (int16_t)__float2int_rn(l);
            else if (int_bytes == 8) static_cast<double*>(out_int)[e] = (double)l;
            else static_cast<int32_t*>(out_int)[e] = __float2int_rn(l);
        }
        if (out_f32) out_f32[e] = l;
    }
    if (uncoded) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) err += __shfl_xor_sync(0xffffffffu, err, o);
        if ((threadIdx.x & 31) == 0 && err) atomicAdd(uncoded, err);
    }
}

// LDPC_count_errors on packed hard decisions: one warp per codeword.
__global__ void count_errors_kernel(const uint32_t* hard, long long n, const uint32_t* ref, long long ref_period,
                                    int hard_words, int kbits, int z, int num_par, unsigned long long* counters) {
    const int lane = threadIdx.x & 31;
    unsigned long long cwe = 0, be = 0;
    const long long nwarps_total = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long i = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += nwarps_total) {
        const uint32_t* h = hard + i * hard_words;
        const uint32_t* r = ref + (i % ref_period) * hard_words;
        unsigned slots = 0;
        unsigned long long bits = 0;
        for (int w = lane; w < hard_words; w += 32) {
            uint32_t d = h[w] ^ r[w];
            const int lo = w * 32;
            if (lo + 32 > kbits) d &= (1u << (kbits - lo)) - 1u;
            bits += __popc(d);
            while (d) {
                const int b = __ffs(d) - 1;
                d &= d - 1;
                slots |= 1u << (((lo + b) % z) % num_par);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bits += __shfl_xor_sync(0xffffffffu, bits, o);
        slots = __reduce_or_sync(0xffffffffu, slots);
        if (bits) {
            be += bits;
            cwe += __popc(slots);
        }
    }
    if (lane == 0) {
        if (cwe) atomicAdd(counters + 0, cwe);
        if (be) atomicAdd(counters + 1, be);
    }
}

}  // namespace ldpc
