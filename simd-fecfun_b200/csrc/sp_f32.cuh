// Layered float decoders: sum-product (tanh / product tree / 2 atanh) and
// offset min-sum, in float (bit-exact with the reference's SIMD_ELEM_BW=-32
// builds LDPCtop_Vec16f_prod / Vec16f_min) and in double (the SIMD_ELEM_BW=-64
// builds LDPCtop_Vec8d_prod / Vec8d_min):
//   Q = P - R                                  decode_functions.cpp:53
//   a = max(|Q| - beta, 0)                     :56-62
//   x = tanh(a/2) (sum-product) or a           min_find.pl:37-41
//   f_j = combine over k != j, fixed tree      min_find.pl:52-164 (gen_trees.cuh)
//         clamped at Max_val, then 2 atanh(.)  min_find.pl:99-107, 44-45
//   R' = f_j with the sign of prod_{k!=j} Q_k  decode_functions.cpp:85-87
//   P  = Q + R'                                :91
// with the same operations in the same order as the oracle (no fused
// multiply-adds; tanh/atanh from ldpc_math.h), so posteriors agree bit for bit.
//
// Work layout: G codewords per CTA, one per group of Z threads (thread
// (t, g) = check row t of every layer).  Posteriors in shared memory, check
// messages in shared memory (RSMEM) or, for large codes, in a global scratch
// area; the layer loop runs over run-time tables, so any code shape works.
// The iteration boundary (syndrome, write-out, refill from a prefetched
// staging buffer) follows the int8 kernel.  Codes whose posteriors and
// staging do not both fit shared memory (double, 5G NR base graph 1 at large
// Z) run without the staging buffer (tb.nostage): a finished codeword's slot
// is refilled straight from global memory.
#pragma once
#include <stdint.h>

#include "gen_trees.cuh"
#include "ldpc_math.h"
#include "tables.h"
#include "writeout.cuh"

namespace ldpc {

__device__ __forceinline__ int sp_wrap(int t, int s, int z) { return (int)min((unsigned)(t + s), (unsigned)(t + s - z)); }

__device__ __forceinline__ void sp_cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void sp_cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void sp_cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}

// element operations of the float and double decoders: IEEE round to nearest,
// never contracted into fused multiply-adds
__device__ __forceinline__ float sp_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sp_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sp_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sp_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sp_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double sp_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float sp_abs(float a) { return fabsf(a); }
__device__ __forceinline__ double sp_abs(double a) { return fabs(a); }
__device__ __forceinline__ float sp_tanh(float a) { return lm_tanh(a); }
__device__ __forceinline__ double sp_tanh(double a) { return lmd_tanh(a); }
__device__ __forceinline__ float sp_atanh(float a) { return lm_atanh(a); }
__device__ __forceinline__ double sp_atanh(double a) { return lmd_atanh(a); }
// the 32-bit word that holds the sign (bit 31)
__device__ __forceinline__ uint32_t sp_signw(float v) { return __float_as_uint(v); }
__device__ __forceinline__ uint32_t sp_signw(double v) { return (uint32_t)__double2hiint(v); }
// v with its sign flipped where bit 31 of sg is set (sign_combine)
__device__ __forceinline__ float sp_flip(float v, uint32_t sg) { return __uint_as_float(__float_as_uint(v) ^ sg); }
__device__ __forceinline__ double sp_flip(double v, uint32_t sg) {
    return __hiloint2double(__double2hiint(v) ^ (int)sg, __double2loint(v));
}

template <class T>
__device__ __forceinline__ void sp_prefetch(T* stage, const T* llr, long long cw, int n, int lane) {
    constexpr int V = 16 / (int)sizeof(T);   // elements per 16-byte copy
    const T* src = llr + cw * (long long)n;
    const unsigned long long base = reinterpret_cast<unsigned long long>(src);
    if ((n % V) == 0 && (base & 15) == 0) {
        for (int i = V * lane; i < n; i += 32 * V) sp_cp_async16(stage + i, src + i);
    } else if (sizeof(T) == 8) {
        for (int i = lane; i < n; i += 32) sp_cp_async8(stage + i, src + i);
    } else {
        for (int i = lane; i < n; i += 32) sp_cp_async4(stage + i, src + i);
    }
}

// Decode codewords [lo, hi) of job with the CTA: the whole decoder; sm_f is
// the CTA's dynamic shared memory (16-byte aligned) for posteriors, staging
// and (RSMEM) messages, r_cta its global message area otherwise.  T = float
// or double.
template <int DMAX, bool PROD, bool RSMEM, class T>
__device__ __forceinline__ void sp_decode_range(const SpTables& tb, const SpJobT<T>& job, long long lo, long long hi,
                                                T* sm_f, T* r_cta) {
    constexpr int V = 16 / (int)sizeof(T);
    __shared__ long long s_cur[32];
    __shared__ long long s_next[32];
    __shared__ int s_it[32];
    __shared__ uint32_t s_synd[2];        // bit g: a check of group g's codeword fails (per iteration parity)
    __shared__ uint32_t s_zero[2];        // bit g: clear group g's messages
    __shared__ int s_busy[2];
    __shared__ unsigned long long s_head;
    __shared__ unsigned long long s_cnt[OMS_MAX_BUCKETS][4];

    const int z = tb.z, n = tb.n, G = tb.G, stride = tb.stride;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
    const int nthr = blockDim.x;
    const int t = tid / G, g = tid - (tid / G) * G;
    const bool active = t < z;
    const int gbase = g * stride;
    const bool staged = !tb.nostage;
    T* Ps = sm_f;
    T* stage = sm_f + ((G * stride + V - 1) & ~(V - 1));            // [G][nstage], 16-byte aligned
    const int nstage = (n + V - 1) & ~(V - 1);
    T* Rbase = RSMEM ? stage + (staged ? G * nstage : 0) : r_cta;
    // check messages: in shared memory each thread's E values are contiguous
    // at an odd stride (E | 1: a warp's lanes fall in distinct banks), so edge
    // e is the thread's base plus e; the global scratch keeps edge-major
    // values (coalesced), edge e at Rt[e * nthr]
    const int rstride = RSMEM ? 1 : nthr;
    T* Rt = RSMEM ? Rbase + tid * (tb.E | 1) : Rbase + tid;
    const T beta = job.beta, maxv = job.maxv;

    for (int i = tid; i < OMS_MAX_BUCKETS * 4; i += nthr) (&s_cnt[0][0])[i] = 0;
    for (int i = tid; i < G * stride; i += nthr) Ps[i] = T(0);
    for (int e = 0; e < tb.E; ++e) Rt[e * rstride] = T(0);
    if (tid < 32) {
        const long long c0 = lo + tid, c1 = lo + G + tid;
        s_cur[tid] = tid < G && c0 < hi ? c0 : -1;
        s_next[tid] = tid < G && c1 < hi ? c1 : -1;
        s_it[tid] = 0;
    }
    if (tid < 2) { s_synd[tid] = 0; s_zero[tid] = 0; s_busy[tid] = 0; }
    if (tid == 0) s_head = (unsigned long long)(lo + 2 * G);
    __syncthreads();
    for (int k = warp; k < G; k += nwarps) {
        if (s_cur[k] >= 0) {
            const T* src = job.llr + s_cur[k] * (long long)n;
            for (int i = lane; i < n; i += 32) Ps[k * stride + i] = src[i];
        }
        if (staged && s_next[k] >= 0) sp_prefetch(stage + k * nstage, job.llr, s_next[k], n, lane);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    __syncthreads();

    auto comb = [](T a, T b) { return PROD ? sp_mul(a, b) : (a < b ? a : b); };
    auto clampf = [maxv](T v) { return maxv < v ? maxv : v; };

    for (int par = 0;; par ^= 1) {
        // ================= one layered iteration =================
        for (int l = 0; l < tb.L; ++l) {
            if (active) {
                const int d = tb.rw[l], eb = tb.ebase[l];
                T q[DMAX], x[DMAX], f[DMAX];
                int addr[DMAX];
                uint32_t rx = 0;
#pragma unroll
                for (int j = 0; j < DMAX; ++j) {
                    if (j < d) {
                        const int e = eb + j;
                        addr[j] = gbase + tb.colz[e] + sp_wrap(t, tb.shift[e], z);
                        const T Q = sp_sub(Ps[addr[j]], Rt[e * rstride]);
                        q[j] = Q;
                        T a = sp_sub(sp_abs(Q), beta);
                        a = a > T(0) ? a : T(0);
                        x[j] = PROD ? sp_tanh(sp_mul(a, T(0.5))) : a;
                        rx ^= sp_signw(Q);
                    }
                }
                run_tree<DMAX>(d, x, f, comb, clampf);
#pragma unroll
                for (int j = 0; j < DMAX; ++j) {
                    if (j < d) {
                        const T fj = PROD ? sp_mul(T(2), sp_atanh(f[j])) : f[j];
                        const uint32_t sg = (rx ^ sp_signw(q[j])) & 0x80000000u;
                        const T rn = sp_flip(fj, sg);
                        Ps[addr[j]] = sp_add(q[j], rn);
                        Rt[(eb + j) * rstride] = rn;
                    }
                }
            }
            __syncthreads();
        }
        if (tid == 0) { s_synd[par ^ 1] = 0; s_zero[par ^ 1] = 0; s_busy[par ^ 1] = 0; }

        // ================= syndrome (early exit once this codeword fails) =================
        if (active) {
            for (int l = 0; l < tb.L; ++l) {
                if (*reinterpret_cast<volatile uint32_t*>(&s_synd[par]) & (1u << g)) break;
                const int d = tb.rw[l], eb = tb.ebase[l];
                uint32_t xr = 0;
                for (int j = 0; j < d; ++j) {
                    const int e = eb + j;
                    xr ^= sp_signw(Ps[gbase + tb.colz[e] + sp_wrap(t, tb.shift[e], z)]);
                }
                if (xr & 0x80000000u) {
                    atomicOr(&s_synd[par], 1u << g);
                    break;
                }
            }
        }
        __syncthreads();

        // ====== each warp: its codewords -- decide, write out, promote, claim, prefetch ======
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncwarp();
        for (int k = warp; k < G; k += nwarps) {
            const long long cw = s_cur[k];
            if (cw < 0) continue;
            const int it = s_it[k] + 1;
            const bool done = !(s_synd[par] & (1u << k)) || it >= job.max_iter;
            if (!done) {
                if (lane == 0) { s_it[k] = it; s_busy[par] = 1; }
                continue;
            }
            const T* pk = Ps + k * stride;
            const uint32_t* ref = job.ref_bits ? job.ref_bits + (cw % job.ref_period) * tb.hard_words : nullptr;
            unsigned errw, errslots;
            warp_hard_decisions<true>([&](int i) { return pk[i] < T(0); }, tb.kbits, tb.hard_words, z, job.num_par,
                                job.hard_out ? job.hard_out + cw * tb.hard_words : nullptr, ref, lane, errw, errslots);
            if (job.post_out) {
                T* dst = job.post_out + cw * (long long)n;
                for (int i = lane; i < n; i += 32) dst[i] = pk[i];
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
                const T* st = staged ? stage + k * nstage : job.llr + nxt * (long long)n;
                for (int i = lane; i < n; i += 32) Ps[k * stride + i] = st[i];
                __syncwarp();
                unsigned long long c = 0;
                if (lane == 0) c = atomicAdd(&s_head, 1ull);
                c = __shfl_sync(0xffffffffu, c, 0);
                const long long fresh = (long long)c < hi ? (long long)c : -1;
                if (staged && fresh >= 0) sp_prefetch(stage + k * nstage, job.llr, fresh, n, lane);
                if (lane == 0) { s_next[k] = fresh; s_busy[par] = 1; }
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
            for (int e = 0; e < tb.E; ++e) Rt[e * rstride] = T(0);
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

// Register budget of a float kernel instance.  Sum-product on rows of weight
// <= 8 with its check messages in global scratch is held to 80 registers
// (no spills): 128-thread CTAs then fit 6 per SM instead of 5 and 384-thread
// CTAs 2 instead of 1, which pays in this latency-bound case (tanh/atanh
// chains).  Every other instance keeps the 128 that a 512-thread CTA allows.
__host__ __device__ constexpr int sp_max_regs(int dmax, bool prod, bool rsmem) {
    return dmax == 8 && prod && !rsmem ? 80 : 128;
}

template <int DMAX, bool PROD, bool RSMEM, int MAXT>
__global__ void __maxnreg__(sp_max_regs(DMAX, PROD, RSMEM)) sp_f32_kernel(const __grid_constant__ SpTables tb, const __grid_constant__ SpJob job) {
    extern __shared__ __align__(16) float sm_f[];
    const long long lo = job.ncw * blockIdx.x / gridDim.x, hi = job.ncw * (blockIdx.x + 1) / gridDim.x;
    sp_decode_range<DMAX, PROD, RSMEM>(tb, job, lo, hi, sm_f,
                                       RSMEM ? nullptr : job.r_scratch + (long long)blockIdx.x * tb.E * blockDim.x);
}

template <int DMAX, bool PROD, bool RSMEM, int MAXT>
__global__ void __launch_bounds__(MAXT) sp_f64_kernel(const __grid_constant__ SpTables tb,
                                                      const __grid_constant__ SpJobT<double> job) {
    extern __shared__ __align__(16) double sm_d[];
    const long long lo = job.ncw * blockIdx.x / gridDim.x, hi = job.ncw * (blockIdx.x + 1) / gridDim.x;
    sp_decode_range<DMAX, PROD, RSMEM>(tb, job, lo, hi, sm_d,
                                       RSMEM ? nullptr : job.r_scratch + (long long)blockIdx.x * tb.E * blockDim.x);
}

}  // namespace ldpc
