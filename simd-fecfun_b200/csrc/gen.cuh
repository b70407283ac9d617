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
// so samples reach ~9.4 sigma (the reference's generator reaches ~9.3 sigma,
// docs/WGN/norm.dist.methods.html).  The same noise is reused for every SNR
// point, as the reference's inner loop does (src/Top/LDPCtop.cpp:89-97).
#pragma once
#include <stdint.h>

#include "tables.h"

namespace ldpc {

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

__device__ __forceinline__ uint4 philox_at(uint64_t seed, uint64_t cw, uint32_t block, uint32_t stream) {
    return philox4x32_10(make_uint4((uint32_t)cw, (uint32_t)(cw >> 32), block, stream),
                         make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
}

// One Box-Muller pair from two 32-bit words (and a refinement word pair for the tail).
__device__ __forceinline__ float2 box_muller(uint32_t w_r, uint32_t w_a, uint64_t seed, uint64_t cw, uint32_t block,
                                             int which) {
    float u1;
    if (w_r < 256u) {
        const uint4 x = philox_at(seed, cw, block, 2u);
        const uint32_t w2 = which ? x.z : x.x;
        u1 = fmaf((float)w_r, 0x1p-32f, fmaf((float)w2, 0x1p-64f, 0x1p-65f));
    } else {
        u1 = fmaf((float)w_r, 0x1p-32f, 0x1p-33f);
    }
    const float r = sqrtf(-2.0f * logf(u1));
    float s, c;
    sincospif((float)w_a * 0x1p-31f, &s, &c);   // angle 2*pi*w_a/2^32
    return make_float2(r * c, r * s);
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
                const int col = tb.term_col[first + q];
                int p = 32 * k + tb.term_shift[first + q];
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

__global__ void __launch_bounds__(256) gen_kernel(const __grid_constant__ GenTables tb, const __grid_constant__ GenJob job) {
    extern __shared__ uint32_t sm[];
    __shared__ unsigned long long s_unc[GEN_MAX_SNR];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpw = gen_warp_words(tb.kbits, tb.mcol, tb.z, tb.n);
    uint32_t* data = sm + warp * wpw;
    uint32_t* cols = data + (tb.kbits / 32 + 2);
    uint32_t* cwbits = cols + tb.mcol * ((tb.z + 31) / 32 + 1);
    for (int i = threadIdx.x; i < GEN_MAX_SNR; i += blockDim.x) s_unc[i] = 0;
    __syncthreads();
    unsigned long long unc[GEN_MAX_SNR];
#pragma unroll
    for (int s = 0; s < GEN_MAX_SNR; ++s) unc[s] = 0;

    const long long nwarps_total = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long i = (long long)blockIdx.x * (blockDim.x >> 5) + warp; i < job.n_per_snr; i += nwarps_total) {
        const uint64_t cw = job.cw_offset + (uint64_t)i;
        draw_data_warp(tb, job.seed, cw, data, lane);
        if (job.data_bits)
            for (int w = lane; w < tb.hard_words; w += 32) job.data_bits[i * tb.hard_words + w] = data[w];
        encode_warp(tb, data, cols, cwbits, lane);
        // noise + LLRs, 4 bits per lane per Philox block
        for (int b = lane; 4 * b < tb.n; b += 32) {
            const uint4 x = philox_at(job.seed, cw, (uint32_t)b, 1u);
            const float2 g0 = box_muller(x.x, x.y, job.seed, cw, (uint32_t)b, 0);
            const float2 g1 = box_muller(x.z, x.w, job.seed, cw, (uint32_t)b, 1);
            const float nz[4] = {g0.x, g0.y, g1.x, g1.y};
            const int idx0 = 4 * b;
            const uint32_t bits4 = (stream_bits32(cwbits, idx0)) & 0xfu;
            for (int s = 0; s < job.n_snr; ++s) {
                float l[4];
                uint32_t packed = 0;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int idx = idx0 + q;
                    if (idx < tb.n) {
                        const int pn = tb.any_punct ? tb.punct[idx] : 0;
                        const int fl = tb.any_filler ? tb.filler[idx] : 0;
                        unc[s] += llr_element((bits4 >> q) & 1u, nz[q], job.sigma[s], job.sigma_factor[s], job.max_abs,
                                              pn, fl, &l[q]);
                        packed |= (uint32_t)(uint8_t)llr_to_i8(l[q]) << (8 * q);
                    }
                }
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
        __syncwarp();
    }
    if (job.uncoded) {
        for (int s = 0; s < job.n_snr; ++s) {
            unsigned long long v = unc[s];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0 && v) atomicAdd(&s_unc[s], v);
        }
        __syncthreads();
        for (int s = threadIdx.x; s < job.n_snr; s += blockDim.x)
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
