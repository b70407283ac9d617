// Layered offset min-sum decoder with the reference's int8 arithmetic, run on
// packed f16x2 lanes (two codewords per 32-bit word).
//
// Reference semantics reproduced bit for bit (src/LDPCDec/decode_functions.cpp:11-103,
// LDPCdecode.cpp:79-201, SIMD_ELEM_BW=8, USE_BETA_OFFSET=1, USE_SAT_ADD_SUB=1):
//   Q   = sat8(P - R)                          decode_functions.cpp:48-51
//   m   = max(wrap8(abs8(Q) - beta8), 0)        :56-61 (abs8(-128) = -128)
//   f_j = min(Max8, min_{k!=j} m_k)             generated min tree, min_find.pl
//   R'  = sign(prod_{k!=j} Q_k) * f_j           :85-87, sign_combine
//   P   = sat8(Q + R')                          :89
// then a syndrome check on the sign bits of P after every iteration; a
// codeword stops when the syndrome is zero or after max_iter iterations
// (LDPCdecode.cpp:172-197).
//
// Why f16x2: every quantity is a small integer (|P| <= 128, |R| <= 127), so
// IEEE half arithmetic on them is exact, and B200 issues packed half2
// min/max at full rate and half2 add at half rate, while the byte-SIMD
// intrinsics (__vsubss4 and friends) are emulated at 8-15 ops/clk/SM.
// Saturation is an explicit clamp to [-128, 127].  The exclusive minimum uses
// min1/min2 of |Q| (tracked before the offset; beta, the clamp at 0 and Max8
// are monotone, so they are applied once per check):
//   f_j = clamp(min1 - beta8, 0, Max8)  if |Q_j| != min1, else clamp(min2 - ...)
// For beta8 = 0 the int8 quirk abs8(-128) = -128 makes that edge's m = 0;
// the BETA0 variant reproduces it.
//
// Work layout (one CTA, persistent):
//   G groups x 2 lanes = 2G codeword slots.  Thread (t, g) = check row t of
//   every layer for group g; tid = t*G + g.  Posteriors of group g live in
//   shared memory at Ps[g*stride + c*Z + v] (stride chosen so a warp's
//   accesses fall in distinct banks).  Check messages R stay in registers,
//   R[l][j] = edge slot j of layer l for this thread's check row.
//   Layers are separated by __syncthreads.  After each iteration a syndrome
//   pass marks converged slots; finished codewords are written out and their
//   slots refilled with the next codeword from a global work counter, so a
//   CTA never idles on codewords that need more iterations than their
//   neighbours.  Results do not depend on which slot decodes a codeword.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

#include <utility>

#include "tables.h"

namespace ldpc {

__device__ __forceinline__ uint32_t h2u(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }
__device__ __forceinline__ __half2 u2h(uint32_t u) { return *reinterpret_cast<__half2*>(&u); }

template <bool BETA0>
__device__ __forceinline__ __half2 abs_q(__half2 q) {
    __half2 a = __habs2(q);
    if (BETA0) {
        // abs8(-128) = -128, and max(-128 - 0, 0) = 0: that edge contributes m = 0
        __half2 is128 = __heq2(q, __float2half2_rn(-128.0f));
        a = __hfma2(is128, __float2half2_rn(-128.0f), a);
    }
    return a;
}

// Shape of the parity-check rows, known at compile time so that the check
// messages R of a thread (one per edge of its check rows) live in registers.
//   FixedShape<rw...>: exact row weights; edge e of layer l is rw[0]+..+rw[l-1]+j.
//   PaddedShape<L,D>: L layers of at most D edges; the weights come from the
//                     tables at run time, edge slot = l*D + j.
template <int... RW>
struct FixedShape {
    static constexpr int L = sizeof...(RW);
    static constexpr int E = (RW + ...);
    static constexpr int D = [] { int m = 0; for (int v : {RW...}) m = v > m ? v : m; return m; }();
    __host__ __device__ static constexpr int maxd(int l) {
        constexpr int rw[] = {RW...};
        return rw[l];
    }
    __host__ __device__ static constexpr int slot(int l, int j) {
        constexpr int rw[] = {RW...};
        int b = 0;
        for (int i = 0; i < l; ++i) b += rw[i];
        return b + j;
    }
    __device__ static bool has(const OmsTables&, int, int) { return true; }
    static constexpr bool fixed = true;
};

template <int L_, int D_>
struct PaddedShape {
    static constexpr int L = L_;
    static constexpr int D = D_;
    static constexpr int E = L_ * D_;
    __host__ __device__ static constexpr int maxd(int) { return D_; }
    __host__ __device__ static constexpr int slot(int l, int j) { return l * D_ + j; }
    __device__ static bool has(const OmsTables& tb, int l, int j) {
        int d = tb.rw[l];
        asm volatile("" : "+r"(d));   // re-read per layer pass instead of keeping L*D predicates live
        return j < d;
    }
    static constexpr bool fixed = false;
};

struct OmsConsts {
    __half2 lo, hi, zero2, beta2, maxv2;
};

// One layer of the layered update for this thread's check row t (all edges
// of the row; the layer index is a template argument so every message
// register index is a compile-time constant).
template <class S, bool BETA0, int l>
__device__ __forceinline__ void oms_layer(const OmsTables& tb, uint32_t* Ps, uint32_t (&R)[S::E], int t, int gbase,
                                          const OmsConsts& k) {
    constexpr int D = S::maxd(l);
    constexpr uint32_t SGN = 0x80008000u;
    const int z = tb.z;
    uint32_t q[D];
    int addr[D];
    __half2 mn1 = __float2half2_rn(1024.0f), mn2 = mn1;
    uint32_t sx = 0;
#pragma unroll
    for (int j = 0; j < D; ++j) {
        if (S::has(tb, l, j)) {
            const int e = S::slot(l, j);
            int v = t + tb.shift[e];
            v = v >= z ? v - z : v;
            addr[j] = gbase + tb.colz[e] + v;
            __half2 Q = __hsub2(u2h(Ps[addr[j]]), u2h(R[e]));
            Q = __hmin2(__hmax2(Q, k.lo), k.hi);
            const __half2 a = abs_q<BETA0>(Q);
            mn2 = __hmin2(mn2, __hmax2(mn1, a));
            mn1 = __hmin2(mn1, a);
            q[j] = h2u(Q);
            sx ^= q[j];
        }
    }
    const __half2 c1 = __hmin2(__hmax2(__hsub2(mn1, k.beta2), k.zero2), k.maxv2);
    const __half2 c2 = __hmin2(__hmax2(__hsub2(mn2, k.beta2), k.zero2), k.maxv2);
    const uint32_t X = h2u(c1) ^ h2u(c2);
    const uint32_t M1 = h2u(c1) ^ (sx & SGN);
#pragma unroll
    for (int j = 0; j < D; ++j) {
        if (S::has(tb, l, j)) {
            const __half2 Q = u2h(q[j]);
            const uint32_t eq = __heq2_mask(abs_q<BETA0>(Q), mn1);
            const uint32_t Rn = M1 ^ (q[j] & SGN) ^ (eq & X);
            __half2 Pn = __hadd2(Q, u2h(Rn));
            Pn = __hmin2(__hmax2(Pn, k.lo), k.hi);
            Ps[addr[j]] = h2u(Pn);
            R[S::slot(l, j)] = Rn;
        }
    }
}

template <class S, bool BETA0, int l>
__device__ __forceinline__ void oms_layer_sync(const OmsTables& tb, uint32_t* Ps, uint32_t (&R)[S::E], int t, int gbase,
                                               bool active, const OmsConsts& k) {
    if (active) oms_layer<S, BETA0, l>(tb, Ps, R, t, gbase, k);
    __syncthreads();
}

template <class S, bool BETA0, int... ls>
__device__ __forceinline__ void oms_iteration(std::integer_sequence<int, ls...>, const OmsTables& tb, uint32_t* Ps,
                                              uint32_t (&R)[S::E], int t, int gbase, bool active, const OmsConsts& k) {
    (oms_layer_sync<S, BETA0, ls>(tb, Ps, R, t, gbase, active, k), ...);
}

// OR over the layers of the XOR of the row's posteriors: sign bits 15/31 set
// when a parity check of lane 0/1 fails.
template <class S, int l>
__device__ __forceinline__ uint32_t oms_row_parity(const OmsTables& tb, const uint32_t* Ps, int t, int gbase) {
    uint32_t x = 0;
#pragma unroll
    for (int j = 0; j < S::maxd(l); ++j) {
        if (S::has(tb, l, j)) {
            const int e = S::slot(l, j);
            int v = t + tb.shift[e];
            v = v >= tb.z ? v - tb.z : v;
            x ^= Ps[gbase + tb.colz[e] + v];
        }
    }
    return x;
}

template <class S, int... ls>
__device__ __forceinline__ uint32_t oms_syndrome(std::integer_sequence<int, ls...>, const OmsTables& tb, const uint32_t* Ps,
                                                 int t, int gbase) {
    return (oms_row_parity<S, ls>(tb, Ps, t, gbase) | ...);
}

template <class S, bool BETA0, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) oms_f16_kernel(const __grid_constant__ OmsTables tb, const __grid_constant__ OmsJob job) {
    extern __shared__ uint32_t Ps[];
    __shared__ long long s_cw[32];       // codeword decoded by slot (-1 = empty)
    __shared__ long long s_fin_cw[32];   // codeword finished at this boundary (-1 = none)
    __shared__ int s_it[32];
    __shared__ int s_fin_it[32];
    __shared__ int s_new[32];            // slot received a new codeword at this boundary
    __shared__ uint32_t s_synd[16];
    __shared__ uint32_t s_zero_mask[16]; // per group: half-lanes whose R must be cleared
    __shared__ int s_continue;
    __shared__ unsigned long long s_cnt[OMS_MAX_BUCKETS][4];

    const int z = tb.z, n = tb.n, G = tb.G, stride = tb.stride;
    const int nslots = 2 * G;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int nwarps = blockDim.x >> 5;
    const int t = tid / G, g = tid - (tid / G) * G;
    const bool active = t < z;
    const int gbase = g * stride;

    for (int i = tid; i < OMS_MAX_BUCKETS * 4; i += blockDim.x) (&s_cnt[0][0])[i] = 0;
    for (int i = tid; i < G * stride; i += blockDim.x) Ps[i] = 0;
    if (tid < 16) { s_synd[tid] = 0; s_zero_mask[tid] = 0; }
    __syncthreads();

    // ---- initial claim: warp 0 takes one codeword per slot
    if (warp == 0) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(job.queue, (unsigned long long)nslots);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (lane < nslots) {
            long long cw = (long long)base + lane;
            s_cw[lane] = cw < job.ncw ? cw : -1;
            s_it[lane] = 0;
            s_new[lane] = cw < job.ncw;
        }
    }
    __syncthreads();

    // ---- load helper: slot k's LLRs into its half-lane of group k>>1
    auto refill = [&](int k) {
        const long long cw = s_cw[k];
        const int gg = k >> 1;
        __half* dst = reinterpret_cast<__half*>(Ps + gg * stride) + (k & 1);
        const int8_t* src = job.llr + cw * (long long)n;
        for (int i = lane; i < n; i += 32) dst[2 * i] = __int2half_rn((int)src[i]);
    };
    for (int k = warp; k < nslots; k += nwarps)
        if (s_new[k]) refill(k);
    __syncthreads();

    uint32_t R[S::E];
#pragma unroll
    for (int e = 0; e < S::E; ++e) R[e] = 0u;

    OmsConsts kc;
    kc.lo = __float2half2_rn(-128.0f);
    kc.hi = __float2half2_rn(127.0f);
    kc.zero2 = __float2half2_rn(0.0f);
    kc.beta2 = u2h(job.beta2);
    kc.maxv2 = u2h(job.maxv2);

    while (true) {
        // ================= one layered iteration =================
        // Per-edge addresses are recomputed every iteration rather than kept
        // live across it (they would need a register per edge): hide t and
        // gbase from loop-invariant code motion.
        int t_it = t, gbase_it = gbase;
        asm volatile("" : "+r"(t_it), "+r"(gbase_it));
        oms_iteration<S, BETA0>(std::make_integer_sequence<int, S::L>(), tb, Ps, R, t_it, gbase_it, active, kc);

        // ================= syndrome of every slot =================
        if (active) {
            const uint32_t acc = oms_syndrome<S>(std::make_integer_sequence<int, S::L>(), tb, Ps, t_it, gbase_it) & 0x80008000u;
            if (acc) atomicOr(&s_synd[g], acc);
        }
        __syncthreads();

        // ================= slot bookkeeping (warp 0) =================
        if (warp == 0) {
            const int k = lane;
            const bool valid = k < nslots;
            long long cw = valid ? s_cw[k] : -1;
            bool done = false;
            int it = 0;
            if (cw >= 0) {
                it = s_it[k] + 1;
                const uint32_t bit = (k & 1) ? 0x80000000u : 0x00008000u;
                done = !(s_synd[k >> 1] & bit) || it >= job.max_iter;
            }
            const unsigned dm = __ballot_sync(0xffffffffu, done);
            unsigned long long base = 0;
            if (dm) {
                if (lane == 0) base = atomicAdd(job.queue, (unsigned long long)__popc(dm));
                base = __shfl_sync(0xffffffffu, base, 0);
            }
            long long ncw_new = -1;
            if (done) {
                const long long c = (long long)base + __popc(dm & ((1u << lane) - 1u));
                ncw_new = c < job.ncw ? c : -1;
            }
            if (valid) {
                s_fin_cw[k] = done ? cw : -1;
                s_fin_it[k] = it;
                s_cw[k] = done ? ncw_new : cw;
                s_it[k] = done ? 0 : it;
                s_new[k] = done && ncw_new >= 0;
            }
            const unsigned busy = __ballot_sync(0xffffffffu, valid && (done ? ncw_new >= 0 : cw >= 0));
            // per group: clear R in half-lanes that finished
            const unsigned dpair = dm >> (2 * (lane & 15));
            if (lane < G) {
                s_zero_mask[lane] = ((dpair & 1u) ? 0x0000ffffu : 0u) | ((dpair & 2u) ? 0xffff0000u : 0u);
                s_synd[lane] = 0;
            }
            if (lane == 0) s_continue = busy != 0;
        }
        __syncthreads();

        // ================= write finished codewords, refill slots =================
        for (int k = warp; k < nslots; k += nwarps) {
            const long long cw = s_fin_cw[k];
            if (cw >= 0) {
                const int gg = k >> 1, hsel = k & 1;
                const __half* src = reinterpret_cast<const __half*>(Ps + gg * stride) + hsel;
                // hard decisions of the data columns, 32 per ballot
                uint32_t mine = 0, errw = 0;
                unsigned errslots = 0;
                const uint32_t* ref = job.ref_bits ? job.ref_bits + (cw % job.ref_period) * tb.hard_words : nullptr;
                for (int w = 0; w < tb.hard_words; ++w) {
                    const int i = w * 32 + lane;
                    bool b = false;
                    if (i < tb.kbits) b = __hlt(src[2 * i], __float2half(0.0f));
                    const uint32_t word = __ballot_sync(0xffffffffu, b);
                    if (lane == (w & 31)) mine = word;
                    if (job.hard_out && ((w & 31) == 31 || w == tb.hard_words - 1) && lane <= (w & 31))
                        job.hard_out[cw * tb.hard_words + (w & ~31) + lane] = mine;
                    if (ref) {
                        const uint32_t rw = ref[w];
                        const bool e = (i < tb.kbits) && (b != (bool)((rw >> lane) & 1u));
                        if (e) errslots |= 1u << ((i % z) % job.num_par);
                        errw += __popc(__ballot_sync(0xffffffffu, e));
                    }
                }
                if (job.post_out) {
                    int8_t* dst = job.post_out + cw * (long long)n;
                    for (int i = lane; i < n; i += 32) dst[i] = (int8_t)__half2int_rn(src[2 * i]);
                }
                if (lane == 0 && job.iters_out) job.iters_out[cw] = (uint8_t)s_fin_it[k];
                if (job.counters) {
                    const unsigned slots = __reduce_or_sync(0xffffffffu, errslots);
                    if (lane == 0) {
                        int b = (int)(cw / job.bucket_size);
                        b = b < job.n_buckets ? b : job.n_buckets - 1;
                        atomicAdd(&s_cnt[b][0], 1ull);
                        atomicAdd(&s_cnt[b][1], (unsigned long long)s_fin_it[k]);
                        if (errw) {
                            atomicAdd(&s_cnt[b][2], (unsigned long long)errw);
                            atomicAdd(&s_cnt[b][3], (unsigned long long)__popc(slots));
                        }
                    }
                }
            }
            __syncwarp();
            if (s_new[k]) refill(k);
        }
        __syncthreads();
        if (active) {
            const uint32_t m = s_zero_mask[g];
            if (m) {
#pragma unroll
                for (int e = 0; e < S::E; ++e) R[e] &= ~m;
            }
        }
        if (!s_continue) break;
    }

    if (job.counters) {
        __syncthreads();
        for (int i = tid; i < job.n_buckets * 4; i += blockDim.x) {
            const unsigned long long v = (&s_cnt[0][0])[i];
            if (v) atomicAdd(job.counters + i, v);
        }
    }
}

}  // namespace ldpc
