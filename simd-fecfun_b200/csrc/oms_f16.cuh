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
//   every layer for group g; tid = g*Z + t.  Posteriors of group g live in
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

#include "codes_fixed.cuh"
#include "tables.h"
#include "writeout.cuh"

namespace ldpc {

// Packed half2 operations on 32-bit registers (inline PTX keeps the two
// lanes in one register; no split into 16-bit halves).
__device__ __forceinline__ uint32_t hsub2(uint32_t a, uint32_t b) { uint32_t d; asm("sub.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); return d; }
__device__ __forceinline__ uint32_t hadd2(uint32_t a, uint32_t b) { uint32_t d; asm("add.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); return d; }
__device__ __forceinline__ uint32_t hmin2(uint32_t a, uint32_t b) { uint32_t d; asm("min.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); return d; }
__device__ __forceinline__ uint32_t hmax2(uint32_t a, uint32_t b) { uint32_t d; asm("max.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); return d; }
__device__ __forceinline__ uint32_t hfma2(uint32_t a, uint32_t b, uint32_t c) { uint32_t d; asm("fma.rn.f16x2 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c)); return d; }
// 0xffff in each lane where a == b, else 0
__device__ __forceinline__ uint32_t heq2_mask(uint32_t a, uint32_t b) { uint32_t d; asm("set.eq.u32.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); return d; }
// 1.0 in each lane where a == b, else 0.0
__device__ __forceinline__ uint32_t heq2(uint32_t a, uint32_t b) { uint32_t d; asm("set.eq.f16x2.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); return d; }
__device__ __forceinline__ uint32_t habs2(uint32_t a) { return a & 0x7fff7fffu; }
// min / max of the magnitudes, with the XOR of the two sign bits as sign:
// one instruction for |.|, the running minimum and the running sign product
__device__ __forceinline__ uint32_t hmin2_xs(uint32_t a, uint32_t b) { uint32_t d; asm("min.xorsign.abs.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); return d; }
__device__ __forceinline__ uint32_t hmax2_xs(uint32_t a, uint32_t b) { uint32_t d; asm("max.xorsign.abs.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); return d; }

constexpr uint32_t H2_M128 = 0xd800d800u;   // -128.0 in both lanes
constexpr uint32_t H2_P127 = 0x57f057f0u;   // +127.0
constexpr uint32_t H2_ZERO = 0u;
constexpr uint32_t H2_1024 = 0x64006400u;   // 1024.0

template <bool BETA0>
__device__ __forceinline__ uint32_t abs_q(uint32_t q) {
    uint32_t a = habs2(q);
    if (BETA0) {
        // abs8(-128) = -128, and max(-128 - 0, 0) = 0: that edge contributes m = 0
        a = hfma2(heq2(q, H2_M128), H2_M128, a);
    }
    return a;
}

// Shape of the parity-check rows, known at compile time so that the check
// messages R of a thread (one per edge of its check rows) live in registers.
//   FixedShape<rw...>: exact row weights; edge e of layer l is rw[0]+..+rw[l-1]+j.
//   PaddedShape<L,D>: L layers of at most D edges; the weights come from the
//                     tables at run time, edge slot = l*D + j.
// Column-local position (t + s) mod z of check t's edge with shift s, with
// t < z and s < z: min over unsigned of (t + s) and (t + s - z).
__device__ __forceinline__ int wrap_add(int t, int s, int z) {
    return (int)min((unsigned)(t + s), (unsigned)(t + s - z));
}

template <int... RW>
struct FixedShape {
    static constexpr int L = sizeof...(RW);
    static constexpr int E = (RW + ...);
    static constexpr int E_REG = E;
    static constexpr int RS_STRIDE = 0;
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
    // shared-memory word of edge e for check row t of a group starting at gbase
    __device__ static int addr(const OmsTables& tb, int e, int t, int gbase) {
        return gbase + tb.colz[e] + wrap_add(t, tb.shift[e], tb.z);
    }
    static constexpr bool fixed = true;
};

// A code compiled in completely (C = Code11ad12, ...): every column and
// shift is an immediate.
template <class C>
struct CompiledShape {
    static constexpr int L = C::L;
    static constexpr int E = C::E;
    static constexpr int E_REG = C::E;
    static constexpr int RS_STRIDE = 0;
    static constexpr int D = C::D;
    __host__ __device__ static constexpr int maxd(int l) { return C::maxd(l); }
    __host__ __device__ static constexpr int slot(int l, int j) { return C::slot(l, j); }
    __device__ static bool has(const OmsTables&, int, int) { return true; }
    __device__ static int addr(const OmsTables&, int e, int t, int gbase) {
        return gbase + C::col(e) * C::Z + wrap_add(t, C::shift(e), C::Z);
    }
    static constexpr bool fixed = true;
};

// Compiled code with the check messages of edge slots >= EREG kept in shared
// memory instead of registers (fewer registers, more resident warps).  They
// sit at Rs[(e - EREG) * NT + tid], NT = the launch's maximum CTA size, so
// every such address is the thread's base plus an immediate.
template <class C, int EREG, int NT>
struct SplitShape : CompiledShape<C> {
    static constexpr int E_REG = EREG;
    static constexpr int RS_STRIDE = NT;
};

template <int L_, int D_>
struct PaddedShape {
    static constexpr int L = L_;
    static constexpr int D = D_;
    static constexpr int E = L_ * D_;
    static constexpr int E_REG = E;
    static constexpr int RS_STRIDE = 0;
    __host__ __device__ static constexpr int maxd(int) { return D_; }
    __host__ __device__ static constexpr int slot(int l, int j) { return l * D_ + j; }
    __device__ static bool has(const OmsTables& tb, int l, int j) {
        int d = tb.rw[l];
        asm volatile("" : "+r"(d));   // re-read per layer pass instead of keeping L*D predicates live
        return j < d;
    }
    __device__ static int addr(const OmsTables& tb, int e, int t, int gbase) {
        return gbase + tb.colz[e] + wrap_add(t, tb.shift[e], tb.z);
    }
    static constexpr bool fixed = false;
};

struct OmsConsts {
    uint32_t beta2, maxv2;
    uint32_t* Rs;        // shared-memory messages of edge slots >= E_REG: Rs[(e - E_REG) * S::RS_STRIDE]
};

template <class S>
__device__ __forceinline__ uint32_t get_r(const uint32_t (&R)[S::E_REG > 0 ? S::E_REG : 1], const OmsConsts& k, int e) {
    if (e < S::E_REG) return R[e < S::E_REG ? e : 0];
    return k.Rs[(e - S::E_REG) * S::RS_STRIDE];
}
template <class S>
__device__ __forceinline__ void set_r(uint32_t (&R)[S::E_REG > 0 ? S::E_REG : 1], const OmsConsts& k, int e, uint32_t v) {
    if (e < S::E_REG) R[e < S::E_REG ? e : 0] = v;
    else k.Rs[(e - S::E_REG) * S::RS_STRIDE] = v;
}

// The posteriors the last layer writes are final for the iteration (no later
// layer touches them), so the parity of this thread's last-layer row is the
// XOR of the values it just wrote: the update keeps it in `plast` and the
// syndrome neither recomputes those addresses nor reloads them.  Same
// posteriors, same parity bit for bit.  (Keeping the final edges of earlier
// layers as well costs a register each and spills.)
// One layer of the layered update for this thread's check row t (all edges
// of the row; the layer index is a template argument so every message
// register index is a compile-time constant).
template <class S, bool BETA0, int l>
__device__ __forceinline__ void oms_layer(const OmsTables& tb, uint32_t* Ps, uint32_t (&R)[S::E_REG > 0 ? S::E_REG : 1], int t, int gbase,
                                          const OmsConsts& k, uint32_t& plast) {
    constexpr int D = S::maxd(l);
    constexpr uint32_t SGN = 0x80008000u;
    uint32_t q[D];
    int addr[D];
    uint32_t mn1 = H2_1024, mn2 = H2_1024;
    uint32_t sx = 0;
#pragma unroll
    for (int j = 0; j < D; ++j) {
        if (S::has(tb, l, j)) {
            const int e = S::slot(l, j);
            addr[j] = S::addr(tb, e, t, gbase);
            uint32_t Q = hsub2(Ps[addr[j]], get_r<S>(R, k, e));
            Q = hmin2(hmax2(Q, H2_M128), H2_P127);
            if (BETA0) {
                const uint32_t a = abs_q<BETA0>(Q);
                mn2 = hmin2(mn2, hmax2(mn1, a));
                mn1 = hmin2(mn1, a);
                sx ^= Q;
            } else {
                // magnitudes as above; mn1's sign bits accumulate the sign
                // product (Q is never -0: P and R start at +0 and x - x = +0)
                mn2 = hmin2_xs(mn2, hmax2_xs(mn1, Q));
                mn1 = hmin2_xs(mn1, Q);
            }
            q[j] = Q;
        }
    }
    if (!BETA0) {
        sx = mn1;
        mn1 = habs2(mn1);
        mn2 = habs2(mn2);
    }
    const uint32_t c1 = hmin2(hmax2(hsub2(mn1, k.beta2), H2_ZERO), k.maxv2);
    const uint32_t c2 = hmin2(hmax2(hsub2(mn2, k.beta2), H2_ZERO), k.maxv2);
    const uint32_t X = c1 ^ c2;
    const uint32_t M1 = c1 ^ (sx & SGN);
#pragma unroll
    for (int j = 0; j < D; ++j) {
        if (S::has(tb, l, j)) {
            const uint32_t eq = heq2_mask(abs_q<BETA0>(q[j]), mn1);
            const uint32_t Rn = M1 ^ (q[j] & SGN) ^ (eq & X);
            const uint32_t Pn = hmin2(hmax2(hadd2(q[j], Rn), H2_M128), H2_P127);
            Ps[addr[j]] = Pn;
            if (l == S::L - 1) plast ^= Pn;
            set_r<S>(R, k, S::slot(l, j), Rn);
        }
    }
}

template <class S, bool BETA0, int l>
__device__ __forceinline__ void oms_layer_sync(const OmsTables& tb, uint32_t* Ps, uint32_t (&R)[S::E_REG > 0 ? S::E_REG : 1], int t, int gbase,
                                               bool active, const OmsConsts& k, uint32_t& plast) {
    if (active) oms_layer<S, BETA0, l>(tb, Ps, R, t, gbase, k, plast);
    __syncthreads();
}

template <class S, bool BETA0, int... ls>
__device__ __forceinline__ void oms_iteration(std::integer_sequence<int, ls...>, const OmsTables& tb, uint32_t* Ps,
                                              uint32_t (&R)[S::E_REG > 0 ? S::E_REG : 1], int t, int gbase, bool active, const OmsConsts& k,
                                              uint32_t& plast) {
    (oms_layer_sync<S, BETA0, ls>(tb, Ps, R, t, gbase, active, k, plast), ...);
}

// XOR of the row's posteriors (the last layer's from the update): sign bits
// 15/31 set when the parity check of lane 0/1 fails.
template <class S, int l>
__device__ __forceinline__ uint32_t oms_row_parity(const OmsTables& tb, const uint32_t* Ps, int t, int gbase,
                                                   uint32_t plast) {
    if (l == S::L - 1) return plast;
    uint32_t x = 0;
#pragma unroll
    for (int j = 0; j < S::maxd(l); ++j) {
        if (S::has(tb, l, j)) x ^= Ps[S::addr(tb, S::slot(l, j), t, gbase)];
    }
    return x;
}

// Syndrome with early exit: a thread publishes failing parity checks as soon
// as it finds them and stops once both lanes of its group are known to fail
// (the result, "some check of this codeword fails", is the same).
template <class S, int l>
__device__ __forceinline__ void oms_syndrome_step(const OmsTables& tb, const uint32_t* Ps, int t, int gbase,
                                                  uint32_t* synd, uint32_t& seen, bool& stop, uint32_t plast) {
    if (stop) return;
    const uint32_t x = oms_row_parity<S, l>(tb, Ps, t, gbase, plast) & 0x80008000u;
    if (x & ~seen) {
        atomicOr(synd, x);
        seen |= x;
    }
    if (((seen | *reinterpret_cast<volatile uint32_t*>(synd)) & 0x80008000u) == 0x80008000u) stop = true;
}

template <class S, int... ls>
__device__ __forceinline__ void oms_syndrome(std::integer_sequence<int, ls...>, const OmsTables& tb, const uint32_t* Ps,
                                             int t, int gbase, uint32_t* synd, uint32_t plast) {
    uint32_t seen = 0;
    bool stop = false;
    // last layer first: its parity needs no loads
    (oms_syndrome_step<S, S::L - 1 - ls>(tb, Ps, t, gbase, synd, seen, stop, plast), ...);
}

// The same syndrome as a loop over the parameter-block tables: more
// instructions per edge, much less code (the unrolled form is a large share
// of the kernel's instruction footprint).
template <class S>
__device__ __forceinline__ void oms_syndrome_loop(const OmsTables& tb, const uint32_t* Ps, int t, int gbase, uint32_t* synd) {
    uint32_t seen = 0;
    int e0 = 0;
    for (int l = 0; l < tb.L; ++l) {
        const int d = tb.rw[l];
        const int base = S::fixed ? e0 : l * tb.D;
        uint32_t x = 0;
        for (int j = 0; j < d; ++j) x ^= Ps[gbase + tb.colz[base + j] + wrap_add(t, tb.shift[base + j], tb.z)];
        e0 += d;
        x &= 0x80008000u;
        if (x & ~seen) {
            atomicOr(synd, x);
            seen |= x;
        }
        if (((seen | *reinterpret_cast<volatile uint32_t*>(synd)) & 0x80008000u) == 0x80008000u) break;
    }
}

// ---- asynchronous global -> shared copies (prefetch of the next codeword) ----
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Copy codeword cw's n LLR bytes into a staging buffer (16-byte chunks when n
// is a multiple of 16, else 4-byte chunks, else single bytes).
// The staging buffer is 16-byte aligned; the source must be too for the
// wide path (n and the llr base pointer are checked).
__device__ __forceinline__ void prefetch_llr(int8_t* stage, const int8_t* llr, long long cw, int n, int lane) {
    const int8_t* src = llr + cw * (long long)n;
    const unsigned long long base = reinterpret_cast<unsigned long long>(llr);
    if ((n & 15) == 0 && (base & 15) == 0) {
        for (int i = 16 * lane; i < n; i += 512) cp_async16(stage + i, src + i);
    } else if ((n & 3) == 0 && (base & 3) == 0) {
        for (int i = 4 * lane; i < n; i += 128) cp_async4(stage + i, src + i);
    } else {
        for (int i = lane; i < n; i += 32) stage[i] = src[i];
    }
}

template <class S, bool BETA0, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) oms_f16_kernel(const __grid_constant__ OmsTables tb, const __grid_constant__ OmsJob job) {
    // dynamic shared memory: posteriors [G][stride] words, then LLR staging [2G][nstage] bytes
    extern __shared__ uint32_t Ps[];
    __shared__ long long s_cur[32];      // codeword decoded by slot (-1 = none)
    __shared__ long long s_next[32];     // codeword prefetched for the slot (-1 = none)
    // iterations done by slot k (-1 = empty), one copy per iteration parity:
    // the slot phase of parity p reads s_it[p] and writes s_it[p ^ 1], so
    // every warp sees the same slot states while others update them
    __shared__ int s_it[2][32];
    // per iteration parity p: failing-check bits and R-clear masks per group, busy flag
    __shared__ uint32_t s_synd[2][16];
    __shared__ uint32_t s_zero_mask[2][16];
    __shared__ int s_busy[2];
    __shared__ unsigned long long s_head;   // next unclaimed codeword of this CTA's range
    __shared__ unsigned long long s_cnt[OMS_MAX_BUCKETS][4];

    const int z = tb.z, n = tb.n, G = tb.G, stride = tb.stride;
    const int nslots = 2 * G;
    const int nstage = (n + 15) & ~15;
    int8_t* stage_base = reinterpret_cast<int8_t*>(Ps) + ((G * stride * 4 + 15) & ~15);
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int nwarps = blockDim.x >> 5;
    // thread tid = g * z + t: a warp holds consecutive rows of one or two
    // codeword pairs (consecutive posterior words, one bank each); measured
    // 0.5 % faster than interleaving the pairs (tid = t * G + g)
    const int g = tid / z, t = tid - (tid / z) * z;
    const bool active = g < G;
    const int gbase = g * stride;
    // this CTA's contiguous share of the codewords (static: no global atomics)
    const long long lo = job.ncw * blockIdx.x / gridDim.x, hi = job.ncw * (blockIdx.x + 1) / gridDim.x;

    for (int i = tid; i < OMS_MAX_BUCKETS * 4; i += blockDim.x) (&s_cnt[0][0])[i] = 0;
    for (int i = tid; i < G * stride; i += blockDim.x) Ps[i] = 0;
    if (tid < 32) {
        const long long c0 = lo + tid, c1 = lo + nslots + tid;
        const bool ok = tid < nslots;
        s_cur[tid] = ok && c0 < hi ? c0 : -1;
        s_next[tid] = ok && c1 < hi ? c1 : -1;
        s_it[0][tid] = ok && c0 < hi ? 0 : -1;
        s_it[1][tid] = -1;
        if (tid < 16) {
            s_synd[0][tid] = s_synd[1][tid] = 0;
            s_zero_mask[0][tid] = s_zero_mask[1][tid] = 0;
        }
        if (tid < 2) s_busy[tid] = 0;
    }
    if (tid == 0) s_head = (unsigned long long)(lo + 2 * nslots);
    __syncthreads();

    // first round: through the staging buffers (16-byte copies) into the
    // posteriors, then prefetch the second round (each warp its own slots)
    for (int k = warp; k < nslots; k += nwarps)
        if (s_cur[k] >= 0) prefetch_llr(stage_base + k * nstage, job.llr, s_cur[k], n, lane);
    cp_async_commit();
    cp_async_wait_all();
    __syncwarp();
    for (int k = warp; k < nslots; k += nwarps) {
        if (s_cur[k] >= 0) {
            __half* dst = reinterpret_cast<__half*>(Ps + (k >> 1) * stride) + (k & 1);
            const int8_t* st = stage_base + k * nstage;
            for (int i = lane; i < n; i += 32) dst[2 * i] = __int2half_rn((int)st[i]);
        }
        __syncwarp();
        if (s_next[k] >= 0) prefetch_llr(stage_base + k * nstage, job.llr, s_next[k], n, lane);
    }
    cp_async_commit();
    __syncthreads();

    uint32_t R[S::E_REG > 0 ? S::E_REG : 1];
#pragma unroll
    for (int e = 0; e < (S::E_REG > 0 ? S::E_REG : 1); ++e) R[e] = 0u;

    OmsConsts kc;
    kc.beta2 = job.beta2;
    kc.maxv2 = job.maxv2;
    // shared-memory messages after the LLR staging area
    kc.Rs = reinterpret_cast<uint32_t*>(stage_base + 2 * G * nstage) + tid;
    for (int e = S::E_REG; e < S::E; ++e) kc.Rs[(e - S::E_REG) * S::RS_STRIDE] = 0u;

    for (int par = 0;; par ^= 1) {
        // ================= one layered iteration =================
        // Per-edge addresses are recomputed every iteration rather than kept
        // live across it (they would need a register per edge): hide t and
        // gbase from loop-invariant code motion.
        int t_it = t, gbase_it = gbase;
        asm volatile("" : "+r"(t_it), "+r"(gbase_it));
        uint32_t plast = 0u;   // XOR of the posteriors the last layer writes
        oms_iteration<S, BETA0>(std::make_integer_sequence<int, S::L>(), tb, Ps, R, t_it, gbase_it, active, kc, plast);
        // (the layer loop ends with a barrier) buffers of the other parity are free again
        if (tid < 16) {
            s_synd[par ^ 1][tid] = 0;
            s_zero_mask[par ^ 1][tid] = 0;
        }
        if (tid == 0) s_busy[par ^ 1] = 0;

        // ================= syndrome of every slot =================
        if (active) {
            if (job.synd_loop) oms_syndrome_loop<S>(tb, Ps, t_it, gbase_it, &s_synd[par][g]);
            else oms_syndrome<S>(std::make_integer_sequence<int, S::L>(), tb, Ps, t_it, gbase_it, &s_synd[par][g], plast);
        }
        __syncthreads();

        // ====== slot phase: decide, write out, promote, claim, prefetch ======
        cp_async_wait_all();   // this warp's prefetches (issued an iteration ago)
        __syncwarp();
        // Lane k of every warp evaluates slot k; the finished slots are dealt
        // out in slot order, the j-th to warp j mod nwarps, so two codewords
        // finishing together go to different warps.
        unsigned done_mask;
        {
            const int itk = lane < nslots ? s_it[par][lane] : -1;
            const bool live = itk >= 0;
            const uint32_t bit = (lane & 1) ? 0x80000000u : 0x00008000u;
            const bool dn = live && (!(s_synd[par][lane >> 1] & bit) || itk + 1 >= job.max_iter);
            done_mask = __ballot_sync(0xffffffffu, dn);
            if (warp == 0 && lane < nslots && !dn) {
                s_it[par ^ 1][lane] = live ? itk + 1 : -1;
                if (live) s_busy[par] = 1;
            }
            // no codeword finished and some slot is live: nothing below changes
            // what the next iteration reads (its first layer barrier orders the
            // s_it writes above), so the phase's barrier is skipped
            if (done_mask == 0 && __any_sync(0xffffffffu, live)) continue;
        }
        int j = 0;
        for (unsigned m = done_mask; m; m &= m - 1, ++j) {
            if (j % nwarps != warp) continue;
            const int k = __ffs(m) - 1;
            const long long cw = s_cur[k];
            const int gg = k >> 1, hsel = k & 1;
            const int it = s_it[par][k] + 1;
            __half* pk = reinterpret_cast<__half*>(Ps + gg * stride) + hsel;
            // hard decisions of the data columns, 32 per ballot; error counts
            const uint32_t* ref = job.ref_bits ? job.ref_bits + (cw % job.ref_period) * tb.hard_words : nullptr;
            unsigned errw, errslots;
            warp_hard_decisions<false>([&](int i) { return __hlt(pk[2 * i], __float2half(0.0f)); }, tb.kbits, tb.hard_words, z,
                                job.num_par, job.hard_out ? job.hard_out + cw * tb.hard_words : nullptr, ref, lane, errw,
                                errslots);
            if (job.post_out) {
                int8_t* dst = job.post_out + cw * (long long)n;
                for (int i = lane; i < n; i += 32) dst[i] = (int8_t)__half2int_rn(pk[2 * i]);
            }
            if (lane == 0 && job.iters_out) job.iters_out[cw] = (uint8_t)it;
            if (job.counters && lane == 0) {
                int bk = (int)(cw / job.bucket_size);
                bk = bk < job.n_buckets ? bk : job.n_buckets - 1;
                atomicAdd(&s_cnt[bk][0], 1ull);
                atomicAdd(&s_cnt[bk][1], (unsigned long long)it);
                if (errw) {
                    atomicAdd(&s_cnt[bk][2], (unsigned long long)errw);
                    atomicAdd(&s_cnt[bk][3], (unsigned long long)__popc(errslots));
                }
            }
            __syncwarp();
            // promote the prefetched codeword, claim and prefetch the one after it
            const long long nxt = s_next[k];
            if (nxt >= 0) {
                const int8_t* st = stage_base + k * nstage;
                for (int i = lane; i < n; i += 32) pk[2 * i] = __int2half_rn((int)st[i]);
                __syncwarp();
                unsigned long long c = 0;
                if (lane == 0) c = atomicAdd(&s_head, 1ull);
                c = __shfl_sync(0xffffffffu, c, 0);
                const long long fresh = (long long)c < hi ? (long long)c : -1;
                if (fresh >= 0) prefetch_llr(stage_base + k * nstage, job.llr, fresh, n, lane);
                if (lane == 0) {
                    s_next[k] = fresh;
                    s_busy[par] = 1;
                }
            }
            if (lane == 0) {
                s_cur[k] = nxt;
                s_it[par ^ 1][k] = nxt >= 0 ? 0 : -1;
                atomicOr(&s_zero_mask[par][gg], hsel ? 0xffff0000u : 0x0000ffffu);
            }
        }
        cp_async_commit();
        __syncthreads();
        if (active) {
            const uint32_t m = s_zero_mask[par][g];
            if (m) {
#pragma unroll
                for (int e = 0; e < S::E_REG; ++e) R[e] &= ~m;
                for (int e = S::E_REG; e < S::E; ++e) kc.Rs[(e - S::E_REG) * S::RS_STRIDE] &= ~m;
            }
        }
        if (!s_busy[par]) break;
    }
    cp_async_wait_all();

    if (job.counters) {
        __syncthreads();
        for (int i = tid; i < job.n_buckets * 4; i += blockDim.x) {
            const unsigned long long v = (&s_cnt[0][0])[i];
            if (v) atomicAdd(job.counters + i, v);
        }
    }
}

}  // namespace ldpc
