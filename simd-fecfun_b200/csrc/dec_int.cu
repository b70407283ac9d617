// Host side of the int16 / int32 offset min-sum decoders (the reference's
// LDPCtop_Vec32s_min and LDPCtop_Vec16w_min builds).
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "internal.h"
#include "oms_int.cuh"

namespace ldpc {

namespace {
typedef void (*int_fn)(const SpTables, const IntJob);
struct IntVariant {
    int bits, dmax;
    bool rsmem;
    int_fn k;
};
#define IV(T_, D_) {8 * (int)sizeof(T_), D_, true, oms_int_kernel<T_, D_, true>}, {8 * (int)sizeof(T_), D_, false, oms_int_kernel<T_, D_, false>}
const IntVariant kInt[] = {IV(int16_t, 8), IV(int16_t, 16), IV(int16_t, 32), IV(int32_t, 8), IV(int32_t, 16), IV(int32_t, 32)};
#undef IV
constexpr int kIntMaxThreads = 512;
}  // namespace

int setup_int(ldpc_ctx* x) {
    const ldpc_code& c = x->code;
    const int bits = x->cfg.variant == LDPC_INT16_OMS ? 16 : 32;
    const int es = bits / 8;
    if (c.mrow > SP_MAX_L || (int)c.row_cols.size() > SP_MAX_E)
        return fail(LDPC_ERR_UNSUPPORTED, "int%d decoder: %d layers / %zu circulants exceed the tables", bits, c.mrow,
                    c.row_cols.size());
    const int dmax = c.max_row_weight <= 8 ? 8 : c.max_row_weight <= 16 ? 16 : c.max_row_weight <= 32 ? 32 : 0;
    if (!dmax) return fail(LDPC_ERR_UNSUPPORTED, "int%d decoder: row weight %d > 32", bits, c.max_row_weight);
    if (c.z > kIntMaxThreads) return fail(LDPC_ERR_UNSUPPORTED, "int%d decoder: Z=%d > %d", bits, c.z, kIntMaxThreads);
    SpTables& t = x->spt;
    memset(&t, 0, sizeof(t));
    t.z = c.z;
    t.mcol = c.mcol;
    t.n = c.z * c.mcol;
    t.L = c.mrow;
    t.kbits = x->kbits;
    t.hard_words = x->hard_words;
    t.E = (int)c.row_cols.size();
    int e0 = 0;
    for (int l = 0; l < c.mrow; ++l) {
        t.rw[l] = (int16_t)c.row_weights[l];
        t.ebase[l] = (int16_t)e0;
        e0 += c.row_weights[l];
    }
    for (int e = 0; e < t.E; ++e) {
        t.colz[e] = c.row_cols[e] * c.z;
        t.shift[e] = (int16_t)c.row_shifts[e];
    }
    int G = std::max(1, std::min(32, 128 / c.z));
    while (G > 1 && ((G * c.z + 31) / 32) * 32 > kIntMaxThreads) --G;
    t.G = G;
    t.stride = t.n + ((((32 + G - 1) / G) - t.n) % 32 + 32) % 32;
    const int threads = ((G * c.z + 31) / 32) * 32;
    const size_t nstage_bytes = ((size_t)t.n * es + 15) & ~(size_t)15;
    const size_t base = ((((size_t)G * t.stride + 3) & ~(size_t)3) * 4) + (size_t)G * nstage_bytes;
    const size_t r_smem = (size_t)(t.E | 1) * threads * 4;   // shared: odd per-thread stride
    const size_t r_glob = (size_t)t.E * threads * 4;          // global scratch: edge-major
    const bool rsmem = base + r_smem <= 160 * 1024;
    const size_t smem = base + (rsmem ? r_smem : 0);
    if (smem > (size_t)kSpMaxSmem) return fail(LDPC_ERR_UNSUPPORTED, "int%d decoder: %zu B of shared memory", bits, smem);
    const IntVariant* v = nullptr;
    for (const IntVariant& k : kInt)
        if (k.bits == bits && k.dmax == dmax && k.rsmem == rsmem) v = &k;
    CUDA_TRY(allow_dynamic_smem((const void*)v->k, kSpMaxSmem));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)v->k, threads, smem));
    if (per_sm < 1) return fail(LDPC_ERR_UNSUPPORTED, "int%d decoder: launch does not fit an SM", bits);
    x->int_kernel = (void*)v->k;
    x->int_threads = threads;
    x->int_smem = (int)smem;
    x->int_ctas = per_sm * x->sms;
    if (!rsmem) CUDA_TRY(cudaMalloc(&x->d_int_scratch, (size_t)x->int_ctas * r_glob));
    // decode_row's offset and Max_row_simd in the element type (decode_functions.cpp:27-32, 59-62):
    // the float offset converts by truncation, the clamp is 1 - (CTYPE)max_row_metric for tiny values
    const double lim = bits == 16 ? 32767.0 : 2147483647.0;
    const float b = x->cfg.beta, m = x->cfg.max_row_metric;
    if (!(b >= 0.0f && b <= lim)) return fail(LDPC_ERR_UNSUPPORTED, "int%d decoder: beta=%g outside [0, %g]", bits, b, lim);
    if (!(m > -lim && m <= lim)) return fail(LDPC_ERR_UNSUPPORTED, "int%d decoder: max_row_metric=%g", bits, m);
    x->ibeta = bits == 16 ? (int)(int16_t)b : (int)b;
    x->imaxv = m < 1e-6 ? (int)(1.0 - (double)(bits == 16 ? (int)(int16_t)m : (int)m)) : (bits == 16 ? (int)(int16_t)m : (int)m);
    if (x->imaxv < 0) return fail(LDPC_ERR_UNSUPPORTED, "int%d decoder: negative row clamp %d", bits, x->imaxv);
    return LDPC_OK;
}

int launch_int(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s) {
    if (!x->int_kernel) return fail(LDPC_ERR_INVALID_ARG, "context was not created for an int16/int32 decoder");
    if (a.n == 0) return LDPC_OK;
    IntJob job;
    memset(&job, 0, sizeof(job));
    job.llr = a.llr;
    job.ncw = (long long)a.n;
    job.post_out = a.post;
    job.hard_out = a.hard;
    job.iters_out = a.iters;
    job.ref_bits = a.ref_bits;
    job.ref_period = a.ref_period > 0 ? a.ref_period : 1;
    job.bucket_size = a.bucket_size > 0 ? a.bucket_size : (long long)a.n;
    job.counters = a.counters;
    job.n_buckets = std::max(1, std::min(a.n_buckets, OMS_MAX_BUCKETS));
    job.num_par = x->code.num_par;
    job.max_iter = (int)x->cfg.max_iter;
    job.beta = x->ibeta;
    job.maxv = x->imaxv;
    job.r_scratch = (int32_t*)x->d_int_scratch;
    const long long want = ((long long)a.n + x->spt.G - 1) / x->spt.G;
    const int grid = (int)std::min<long long>(want, x->int_ctas);
    ((int_fn)x->int_kernel)<<<grid, x->int_threads, x->int_smem, s>>>(x->spt, job);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

}  // namespace ldpc
