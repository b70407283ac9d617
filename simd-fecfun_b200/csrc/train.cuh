// Learned-offset float offset min-sum: the layered decoder of the float
// OMS variant (decode_functions.cpp:11-103 with SIMD_ELEM_BW=-32, min tree
// replaced by min1/min2, exact for min) unrolled for a fixed number of
// iterations, with offset beta[it][l] per iteration and layer, and its
// hand-written adjoint.
//
// Loss (the gradient the backward kernel returns):
//   L = sum_it w[it] * inv_norm * sum_cw sum_v softplus(-s_v * P_{it+1}[v]),
//   s_v = 1 - 2 c_v (c = sent code bit), P_{it+1} = posteriors after iteration it.
//
// Forward (oms_train_fwd): one codeword per CTA, thread t = check row t of
// every layer; posteriors P and messages R in shared memory.  At the start
// of every iteration it writes the checkpoint (P_it, R_it); after the last it
// writes P_T.  In evaluation mode it stops a codeword once its syndrome is
// zero (the reference's early exit) and writes results instead.
//
// Backward (oms_train_bwd), per codeword, iterations in reverse:
//   1. gP += dL/dP_{it+1} (loss adjoint);
//   2. reload (P_it, R_it) and recompute the iteration's layers, keeping each
//      edge's Q in the slot of its message (per-iteration checkpoint +
//      recompute);
//   3. layers in reverse: from Q recompute a = |Q| - beta, m = max(a, 0),
//      min1/min2/argmin, the clamp and the signs, then
//        gR'_j = gP[v_j] + gR[e_j]      (P' = Q + R', R' reused next iteration)
//        gf_j  = gR'_j * sign_j          (zero where the clamp is active)
//        gm[argmin1] += sum_{j != argmin1} gf_j,  gm[argmin2] += gf[argmin1]
//        ga_k = gm_k * [a_k > 0];  gbeta[it][l] -= sum ga_k
//        gQ_j = gP[v_j] + ga_j * sign(Q_j)
//        gP[v_j] = gQ_j;  gR[e_j] = -gQ_j  (Q = P - R_previous)
//   gbeta is reduced per CTA in a fixed order (deterministic) into
//   gbeta_part[cta][it*L + l]; the host sums the CTA rows.
#pragma once
#include <stdint.h>

#include "tables.h"

namespace ldpc {

struct TrainJob {
    const float* llr;                // [ncw][n]
    long long ncw;
    int iters;
    const float* beta;               // [iters][L]
    float maxv;                      // row clamp (decode_row's Max_val)
    float* ckpt_p;                   // [iters+1][ncw][n]   (forward writes, backward reads)
    float* ckpt_r;                   // [iters][ncw][E*z]
    const uint8_t* cw_bits;          // [ncw][n] sent code bits (backward)
    const float* loss_w;             // [iters]
    float inv_norm;
    float* gbeta_part;               // [gridDim][iters*L]
    float* grad_llr;                 // [ncw][n] or null
    // evaluation mode (forward only)
    int early_exit;
    uint8_t* iters_out;
    uint32_t* hard_out;
    float* post_out;
};

constexpr int TRAIN_MAX_ITERS = 64;

__device__ __forceinline__ int tr_wrap(int t, int s, int z) { return (int)min((unsigned)(t + s), (unsigned)(t + s - z)); }

// One layer's forward update for check row t; if keep_q, Q replaces the
// message in R (the backward recompute).
template <int DMAX>
__device__ __forceinline__ void tr_layer(const SpTables& tb, int l, float* P, float* R, int t, float beta, float maxv,
                                         bool keep_q) {
    const int d = tb.rw[l], eb = tb.ebase[l], z = tb.z;
    float q[DMAX];
    int addr[DMAX];
    float mn1 = __int_as_float(0x7f800000), mn2 = mn1;
    int idx = 0;
    uint32_t rx = 0;
#pragma unroll
    for (int j = 0; j < DMAX; ++j) {
        if (j < d) {
            const int e = eb + j;
            addr[j] = tb.colz[e] + tr_wrap(t, tb.shift[e], z);
            const float Q = __fsub_rn(P[addr[j]], R[e * z + t]);
            float a = __fsub_rn(fabsf(Q), beta);
            a = a > 0.0f ? a : 0.0f;
            if (a < mn1) {
                mn2 = mn1;
                mn1 = a;
                idx = j;
            } else if (a < mn2) {
                mn2 = a;
            }
            rx ^= __float_as_uint(Q);
            q[j] = Q;
        }
    }
#pragma unroll
    for (int j = 0; j < DMAX; ++j) {
        if (j < d) {
            float f = j == idx ? mn2 : mn1;
            f = maxv < f ? maxv : f;
            const uint32_t sg = (rx ^ __float_as_uint(q[j])) & 0x80000000u;
            const float rn = __uint_as_float(__float_as_uint(f) ^ sg);
            P[addr[j]] = __fadd_rn(q[j], rn);
            R[(eb + j) * z + t] = keep_q ? q[j] : rn;
        }
    }
}

__device__ __forceinline__ bool tr_syndrome_ok(const SpTables& tb, const float* P, int t) {
    bool ok = true;
    for (int l = 0; l < tb.L && ok; ++l) {
        uint32_t x = 0;
        for (int j = 0; j < tb.rw[l]; ++j) {
            const int e = tb.ebase[l] + j;
            x ^= __float_as_uint(P[tb.colz[e] + tr_wrap(t, tb.shift[e], tb.z)]);
        }
        ok = !(x & 0x80000000u);
    }
    return ok;
}

template <int DMAX>
__global__ void __launch_bounds__(512) oms_train_fwd(const __grid_constant__ SpTables tb, const __grid_constant__ TrainJob job) {
    extern __shared__ float tr_sm[];
    __shared__ int s_fail;
    const int n = tb.n, z = tb.z, EZ = tb.E * tb.z;
    float* P = tr_sm;
    float* R = tr_sm + ((n + 3) & ~3);
    const int tid = threadIdx.x, nthr = blockDim.x;
    const bool active = tid < z;
    for (long long cw = blockIdx.x; cw < job.ncw; cw += gridDim.x) {
        __syncthreads();
        const float* src = job.llr + cw * (long long)n;
        for (int i = tid; i < n; i += nthr) P[i] = src[i];
        for (int i = tid; i < EZ; i += nthr) R[i] = 0.0f;
        __syncthreads();
        int it = 0;
        for (; it < job.iters; ++it) {
            if (job.ckpt_p) {
                float* cp = job.ckpt_p + ((long long)it * job.ncw + cw) * n;
                for (int i = tid; i < n; i += nthr) cp[i] = P[i];
                float* cr = job.ckpt_r + ((long long)it * job.ncw + cw) * EZ;
                for (int i = tid; i < EZ; i += nthr) cr[i] = R[i];
                __syncthreads();   // every thread has read P and R before the layers change them
            }
            for (int l = 0; l < tb.L; ++l) {
                if (active) tr_layer<DMAX>(tb, l, P, R, tid, job.beta[it * tb.L + l], job.maxv, false);
                __syncthreads();
            }
            if (job.early_exit) {
                if (tid == 0) s_fail = 0;
                __syncthreads();
                if (active && !tr_syndrome_ok(tb, P, tid)) s_fail = 1;
                __syncthreads();
                if (!s_fail) {
                    ++it;
                    break;
                }
            }
        }
        if (job.ckpt_p) {
            float* cp = job.ckpt_p + ((long long)job.iters * job.ncw + cw) * n;
            for (int i = tid; i < n; i += nthr) cp[i] = P[i];
        }
        if (job.post_out) {
            float* dst = job.post_out + cw * (long long)n;
            for (int i = tid; i < n; i += nthr) dst[i] = P[i];
        }
        if (job.iters_out && tid == 0) job.iters_out[cw] = (uint8_t)min(it, job.iters);
        if (job.hard_out) {
            for (int w = tid; w < tb.hard_words; w += nthr) {
                uint32_t word = 0;
                for (int b = 0; b < 32; ++b) {
                    const int i = w * 32 + b;
                    if (i < tb.kbits && P[i] < 0.0f) word |= 1u << b;
                }
                job.hard_out[cw * tb.hard_words + w] = word;
            }
        }
    }
}

// Global -> shared copy of m floats: 16-byte vector loads, several in flight
// per thread, when both ends are 16-byte aligned and m % 4 == 0.
__device__ __forceinline__ void tr_copy(float* dst, const float* src, int m) {
    const int tid = threadIdx.x, nthr = blockDim.x;
    if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0 && (m & 3) == 0) {
        const float4* s4 = reinterpret_cast<const float4*>(src);
        float4* d4 = reinterpret_cast<float4*>(dst);
        const int m4 = m >> 2;
#pragma unroll 8
        for (int i = tid; i < m4; i += nthr) d4[i] = __ldg(s4 + i);
    } else {
#pragma unroll 8
        for (int i = tid; i < m; i += nthr) dst[i] = __ldg(src + i);
    }
}

// deterministic block sum of v (fixed reduction order); all threads must call
__device__ __forceinline__ float tr_block_sum(float v, float* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    float s = 0.0f;
    for (int w = 0; w < nw; ++w) s += red[w];
    return s;
}

template <int DMAX>
__global__ void __launch_bounds__(512) oms_train_bwd(const __grid_constant__ SpTables tb, const __grid_constant__ TrainJob job) {
    extern __shared__ float tr_sm[];
    __shared__ float s_red[16];
    const int n = tb.n, z = tb.z, EZ = tb.E * tb.z, L = tb.L;
    const int n4 = (n + 3) & ~3, ez4 = (EZ + 3) & ~3;
    float* P = tr_sm;
    float* QR = P + n4;
    float* gP = QR + ez4;
    float* gR = gP + n4;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const bool active = tid < z;
    const int t = tid;
    float* part = job.gbeta_part + (long long)blockIdx.x * job.iters * L;
    for (int i = tid; i < job.iters * L; i += nthr) part[i] = 0.0f;

    for (long long cw = blockIdx.x; cw < job.ncw; cw += gridDim.x) {
        __syncthreads();
        for (int i = tid; i < n; i += nthr) gP[i] = 0.0f;
        for (int i = tid; i < EZ; i += nthr) gR[i] = 0.0f;
        const uint8_t* bits = job.cw_bits + cw * (long long)n;
        for (int it = job.iters - 1; it >= 0; --it) {
            __syncthreads();
            // 1. loss adjoint at the end of iteration it
            const float* pe = job.ckpt_p + ((long long)(it + 1) * job.ncw + cw) * n;
            const float wk = job.loss_w[it] * job.inv_norm;
#pragma unroll 4
            for (int i = tid; i < n; i += nthr) {
                const float s = bits[i] ? -1.0f : 1.0f;
                const float x = -s * pe[i];
                const float sg = 1.0f / (1.0f + __expf(-x));     // d softplus(x)/dx
                gP[i] += wk * (-s) * sg;
            }
            // 2. reload the checkpoint and recompute the layers, keeping Q
            const float* cp = job.ckpt_p + ((long long)it * job.ncw + cw) * n;
            const float* cr = job.ckpt_r + ((long long)it * job.ncw + cw) * EZ;
            tr_copy(P, cp, n);
            tr_copy(QR, cr, EZ);
            __syncthreads();
            for (int l = 0; l < L; ++l) {
                if (active) tr_layer<DMAX>(tb, l, P, QR, t, job.beta[it * L + l], job.maxv, true);
                __syncthreads();
            }
            // 3. layers in reverse
            for (int l = L - 1; l >= 0; --l) {
                const float beta = job.beta[it * L + l];
                float gb = 0.0f;
                if (active) {
                    const int d = tb.rw[l], eb = tb.ebase[l];
                    float q[DMAX], a[DMAX], gq[DMAX], gf[DMAX];
                    int addr[DMAX];
                    float mn1 = __int_as_float(0x7f800000), mn2 = mn1;
                    int i1 = 0, i2 = -1;
                    uint32_t rx = 0;
#pragma unroll
                    for (int j = 0; j < DMAX; ++j) {
                        if (j < d) {
                            const int e = eb + j;
                            addr[j] = tb.colz[e] + tr_wrap(t, tb.shift[e], z);
                            q[j] = QR[e * z + t];
                            a[j] = __fsub_rn(fabsf(q[j]), beta);
                            const float m = a[j] > 0.0f ? a[j] : 0.0f;
                            if (m < mn1) {
                                mn2 = mn1;
                                i2 = i1;
                                mn1 = m;
                                i1 = j;
                            } else if (m < mn2) {
                                mn2 = m;
                                i2 = j;
                            }
                            rx ^= __float_as_uint(q[j]);
                        }
                    }
                    float gm1 = 0.0f, gm2 = 0.0f;   // adjoints of the inputs at i1 and i2
#pragma unroll
                    for (int j = 0; j < DMAX; ++j) {
                        if (j < d) {
                            const int e = eb + j;
                            const float gpost = gP[addr[j]];
                            const float grn = gpost + gR[e * z + t];
                            const float fu = j == i1 ? mn2 : mn1;
                            const bool neg = ((rx ^ __float_as_uint(q[j])) & 0x80000000u) != 0;
                            gf[j] = fu < job.maxv ? (neg ? -grn : grn) : 0.0f;
                            gq[j] = gpost;
                            if (j == i1) gm2 += gf[j];
                            else gm1 += gf[j];
                        }
                    }
#pragma unroll
                    for (int j = 0; j < DMAX; ++j) {
                        if (j < d) {
                            float gm = (j == i1 ? gm1 : 0.0f) + (j == i2 ? gm2 : 0.0f);
                            const float ga = a[j] > 0.0f ? gm : 0.0f;
                            gb -= ga;
                            gq[j] += q[j] < 0.0f ? -ga : ga;
                            gP[addr[j]] = gq[j];
                            gR[(eb + j) * z + t] = -gq[j];
                        }
                    }
                }
                const float s = tr_block_sum(gb, s_red);
                if (tid == 0) part[it * L + l] += s;
                __syncthreads();
            }
        }
        if (job.grad_llr) {
            __syncthreads();
            float* g = job.grad_llr + cw * (long long)n;
            for (int i = tid; i < n; i += nthr) g[i] = gP[i];
        }
    }
}

}  // namespace ldpc
