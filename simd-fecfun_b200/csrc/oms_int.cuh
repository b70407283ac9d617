// Layered offset min-sum with the reference's int16 and int32 element
// semantics (LDPCtop_Vec32s_min, LDPCtop_Vec16w_min: SIMD_ELEM_BW = 16 / 32,
// USE_SAT_ADD_SUB = 1; decode_functions.cpp:11-103, LDPCdecode.cpp:79-201):
//   Q = sat_W(P - R)                       :48-51 (sub_saturated)
//   m = max(wrap_W(abs_W(Q) - beta_W), 0)  :56-61 (abs of the most negative
//                                          value is itself; beta truncated to W bits)
//   f_j = min(Max_W, min_{k!=j} m_k)       generated min tree (exact for integers)
//   R' = sign(prod_{k!=j} Q_k) * f_j       :85-87
//   P = sat_W(Q + R')                      :89 (add_saturated)
// Values are held as sign-extended int32 in shared memory, one codeword per
// group of Z threads (thread (t, g) = check row t of every layer), with the
// run-time tables, slot refill and fused counting of the float decoder.
#pragma once
#include <stdint.h>

#include "sp_f32.cuh"
#include "tables.h"

namespace ldpc {

struct IntJob {
    const void* llr;                 // [ncw][n] TL
    long long ncw;
    void* post_out;                  // [ncw][n] TL or null
    uint32_t* hard_out;
    uint8_t* iters_out;
    const uint32_t* ref_bits;
    long long ref_period;
    long long bucket_size;
    unsigned long long* counters;
    int n_buckets;
    int num_par;
    int max_iter;
    int beta;                        // beta truncated to the element type
    int maxv;                        // Max_row_simd in the element type
    int32_t* r_scratch;              // global check messages when they do not fit shared memory
};

template <int W>
__device__ __forceinline__ int32_t int_sat(int32_t a, int32_t b, bool sub) {
    if (W == 32) {
        int32_t d;
        if (sub) asm("sub.sat.s32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
        else asm("add.sat.s32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
        return d;
    }
    const int32_t v = sub ? a - b : a + b;   // |a|, |b| < 2^15: no int32 overflow
    return min(max(v, -32768), 32767);
}

// wrap to W bits, sign-extended
template <int W>
__device__ __forceinline__ int32_t int_wrap(int32_t v) {
    return W == 32 ? v : (int32_t)(int16_t)(uint16_t)(uint32_t)v;
}

template <int W>
__device__ __forceinline__ int32_t int_abs(int32_t q) {
    // abs of the most negative W-bit value is itself (two's complement wrap)
    return q < 0 ? int_wrap<W>((int32_t)(0u - (uint32_t)q)) : q;
}

template <int W, int DMAX>
__device__ __forceinline__ void int_layer(const SpTables& tb, int l, int32_t* Ps, int32_t* Rt, int rstride, int t,
                                          int gbase, int beta, int maxv) {
    const int d = tb.rw[l], eb = tb.ebase[l], z = tb.z;
    int32_t q[DMAX];
    int addr[DMAX];
    int32_t mn1 = 0x7fffffff, mn2 = 0x7fffffff;
    uint32_t rx = 0;
#pragma unroll
    for (int j = 0; j < DMAX; ++j) {
        if (j < d) {
            const int e = eb + j;
            addr[j] = gbase + tb.colz[e] + sp_wrap(t, tb.shift[e], z);
            const int32_t Q = int_sat<W>(Ps[addr[j]], Rt[e * rstride], true);
            int32_t m = int_wrap<W>(int_abs<W>(Q) - beta);
            m = m > 0 ? m : 0;
            mn2 = min(mn2, max(mn1, m));
            mn1 = min(mn1, m);
            rx ^= (uint32_t)Q;
            q[j] = Q;
        }
    }
    const int32_t f1 = min(maxv, mn1), f2 = min(maxv, mn2);
#pragma unroll
    for (int j = 0; j < DMAX; ++j) {
        if (j < d) {
            int32_t m = int_wrap<W>(int_abs<W>(q[j]) - beta);
            m = m > 0 ? m : 0;
            const int32_t f = m == mn1 ? f2 : f1;
            const int32_t rn = ((rx ^ (uint32_t)q[j]) & 0x80000000u) ? -f : f;
            Ps[addr[j]] = int_sat<W>(q[j], rn, false);
            Rt[(eb + j) * rstride] = rn;
        }
    }
}

// Copy codeword cw's n elements of TL into staging (16-byte chunks when the
// byte count and addresses allow, else 4-byte chunks, else element-wise).
template <class TL>
__device__ __forceinline__ void int_prefetch(TL* stage, const TL* llr, long long cw, int n, int lane) {
    const TL* src = llr + cw * (long long)n;
    const int bytes = n * (int)sizeof(TL);
    const unsigned long long a = reinterpret_cast<unsigned long long>(src);
    char* s = reinterpret_cast<char*>(stage);
    const char* g = reinterpret_cast<const char*>(src);
    if ((bytes & 15) == 0 && (a & 15) == 0) {
        for (int i = 16 * lane; i < bytes; i += 512) sp_cp_async16(s + i, g + i);
    } else if ((bytes & 3) == 0 && (a & 3) == 0) {
        for (int i = 4 * lane; i < bytes; i += 128) sp_cp_async4(s + i, g + i);
    } else {
        for (int i = lane; i < n; i += 32) stage[i] = src[i];
    }
}

template <class TL, int DMAX, bool RSMEM>
__global__ void __launch_bounds__(512) oms_int_kernel(const __grid_constant__ SpTables tb, const __grid_constant__ IntJob job) {
    constexpr int W = 8 * (int)sizeof(TL);
    extern __shared__ __align__(16) int32_t sm_i[];
    __shared__ long long s_cur[32];
    __shared__ long long s_next[32];
    __shared__ int s_it[32];
    __shared__ uint32_t s_synd[2];
    __shared__ uint32_t s_zero[2];
    __shared__ int s_busy[2];
    __shared__ unsigned long long s_head;
    __shared__ unsigned long long s_cnt[OMS_MAX_BUCKETS][4];

    const int z = tb.z, n = tb.n, G = tb.G, stride = tb.stride;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
    const int nthr = blockDim.x;
    const int t = tid / G, g = tid - (tid / G) * G;
    const bool active = t < z;
    const int gbase = g * stride;
    int32_t* Ps = sm_i;
    TL* stage = reinterpret_cast<TL*>(sm_i + ((G * stride + 3) & ~3));        // [G][nstage], 16-byte aligned
    const int nstage = ((n * (int)sizeof(TL) + 15) & ~15) / (int)sizeof(TL);
    int32_t* Rbase = RSMEM ? reinterpret_cast<int32_t*>(stage + G * nstage)
                           : job.r_scratch + (long long)blockIdx.x * tb.E * nthr;
    // check messages: in shared memory each thread's E words are contiguous
    // at an odd stride (E | 1: a warp's lanes fall in distinct banks), so edge
    // e is the thread's base plus e; the global scratch keeps edge-major
    // words (coalesced)
    const int rstride = RSMEM ? 1 : nthr;
    int32_t* Rt = RSMEM ? Rbase + tid * (tb.E | 1) : Rbase + tid;
    const TL* llr = reinterpret_cast<const TL*>(job.llr);
    const long long lo = job.ncw * blockIdx.x / gridDim.x, hi = job.ncw * (blockIdx.x + 1) / gridDim.x;

    for (int i = tid; i < OMS_MAX_BUCKETS * 4; i += nthr) (&s_cnt[0][0])[i] = 0;
    for (int i = tid; i < G * stride; i += nthr) Ps[i] = 0;
    for (int e = 0; e < tb.E; ++e) Rt[e * rstride] = 0;
    if (tid < 32) {
        const long long c0 = lo + tid, c1 = lo + G + tid;
        s_cur[tid] = tid < G && c0 < hi ? c0 : -1;
        s_next[tid] = tid < G && c1 < hi ? c1 : -1;
        s_it[tid] = 0;
    }
    if (tid < 2) {
        s_synd[tid] = 0;
        s_zero[tid] = 0;
        s_busy[tid] = 0;
    }
    if (tid == 0) s_head = (unsigned long long)(lo + 2 * G);
    __syncthreads();
    for (int k = warp; k < G; k += nwarps) {
        if (s_cur[k] >= 0) {
            const TL* src = llr + s_cur[k] * (long long)n;
            for (int i = lane; i < n; i += 32) Ps[k * stride + i] = (int32_t)src[i];
        }
        if (s_next[k] >= 0) int_prefetch(stage + k * nstage, llr, s_next[k], n, lane);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    __syncthreads();

    for (int par = 0;; par ^= 1) {
        for (int l = 0; l < tb.L; ++l) {
            if (active) int_layer<W, DMAX>(tb, l, Ps, Rt, rstride, t, gbase, job.beta, job.maxv);
            __syncthreads();
        }
        if (tid == 0) {
            s_synd[par ^ 1] = 0;
            s_zero[par ^ 1] = 0;
            s_busy[par ^ 1] = 0;
        }
        // syndrome on the sign bits (early exit once this codeword fails)
        if (active) {
            for (int l = 0; l < tb.L; ++l) {
                if (*reinterpret_cast<volatile uint32_t*>(&s_synd[par]) & (1u << g)) break;
                const int d = tb.rw[l], eb = tb.ebase[l];
                uint32_t xr = 0;
                for (int j = 0; j < d; ++j) {
                    const int e = eb + j;
                    xr ^= (uint32_t)Ps[gbase + tb.colz[e] + sp_wrap(t, tb.shift[e], z)];
                }
                if (xr & 0x80000000u) {
                    atomicOr(&s_synd[par], 1u << g);
                    break;
                }
            }
        }
        __syncthreads();

        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncwarp();
        for (int k = warp; k < G; k += nwarps) {
            const long long cw = s_cur[k];
            if (cw < 0) continue;
            const int it = s_it[k] + 1;
            const bool done = !(s_synd[par] & (1u << k)) || it >= job.max_iter;
            if (!done) {
                if (lane == 0) {
                    s_it[k] = it;
                    s_busy[par] = 1;
                }
                continue;
            }
            const int32_t* pk = Ps + k * stride;
            const uint32_t* ref = job.ref_bits ? job.ref_bits + (cw % job.ref_period) * tb.hard_words : nullptr;
            unsigned errw, errslots;
            warp_hard_decisions<true>([&](int i) { return pk[i] < 0; }, tb.kbits, tb.hard_words, z, job.num_par,
                                job.hard_out ? job.hard_out + cw * tb.hard_words : nullptr, ref, lane, errw, errslots);
            if (job.post_out) {
                TL* dst = reinterpret_cast<TL*>(job.post_out) + cw * (long long)n;
                for (int i = lane; i < n; i += 32) dst[i] = (TL)pk[i];
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
            const long long nxt = s_next[k];
            if (nxt >= 0) {
                const TL* st = stage + k * nstage;
                for (int i = lane; i < n; i += 32) Ps[k * stride + i] = (int32_t)st[i];
                __syncwarp();
                unsigned long long c = 0;
                if (lane == 0) c = atomicAdd(&s_head, 1ull);
                c = __shfl_sync(0xffffffffu, c, 0);
                const long long fresh = (long long)c < hi ? (long long)c : -1;
                if (fresh >= 0) int_prefetch(stage + k * nstage, llr, fresh, n, lane);
                if (lane == 0) {
                    s_next[k] = fresh;
                    s_busy[par] = 1;
                }
            }
            if (lane == 0) {
                s_cur[k] = nxt;
                s_it[k] = 0;
                atomicOr(&s_zero[par], 1u << k);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        __syncthreads();
        if (active && (s_zero[par] & (1u << g)))
            for (int e = 0; e < tb.E; ++e) Rt[e * rstride] = 0;
        if (!s_busy[par]) break;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (job.counters) {
        __syncthreads();
        for (int i = tid; i < job.n_buckets * 4; i += nthr) {
            const unsigned long long v = (&s_cnt[0][0])[i];
            if (v) atomicAdd(job.counters + i, v);
        }
    }
}

}  // namespace ldpc
