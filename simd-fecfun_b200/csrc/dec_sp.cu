// Host side of the float decoders (sum-product, offset min-sum).
#include <algorithm>
#include <cstring>

#include "internal.h"
#include "sp_f32.cuh"

namespace ldpc {

namespace {
constexpr int SP_MAXT = 512;
struct SpVariant {
    int dmax;
    bool prod, rsmem;
    sp_fn k;
};
#define SPV(D_, P_, R_) {D_, P_, R_, sp_f32_kernel<D_, P_, R_, SP_MAXT>}
const SpVariant kSp[] = {
    SPV(8, true, true),  SPV(8, true, false),  SPV(8, false, true),  SPV(8, false, false),
    SPV(16, true, true), SPV(16, true, false), SPV(16, false, true), SPV(16, false, false),
    SPV(32, true, true), SPV(32, true, false), SPV(32, false, true), SPV(32, false, false),
};
#undef SPV
}  // namespace

void fill_sp_tables(const ldpc_code& c, int G, SpTables* out) {
    SpTables& t = *out;
    memset(&t, 0, sizeof(t));
    t.z = c.z;
    t.mcol = c.mcol;
    t.n = c.z * c.mcol;
    t.L = c.mrow;
    t.kbits = c.z * (c.mcol - c.mrow);
    t.hard_words = (t.kbits + 31) / 32;
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
    t.G = G;
    t.stride = t.n + ((((32 + G - 1) / G) - t.n) % 32 + 32) % 32;
}

int setup_sp(ldpc_ctx* x) {
    const ldpc_code& c = x->code;
    const bool prod = x->cfg.variant == LDPC_F32_SP;
    if (c.mrow > SP_MAX_L || (int)c.row_cols.size() > SP_MAX_E)
        return fail(LDPC_ERR_UNSUPPORTED, "float decoder: %d layers / %zu edges exceed the tables", c.mrow,
                    c.row_cols.size());
    const int dmax = c.max_row_weight <= 8 ? 8 : c.max_row_weight <= 16 ? 16 : c.max_row_weight <= 32 ? 32 : 0;
    if (!dmax) return fail(LDPC_ERR_UNSUPPORTED, "float decoder: row weight %d > 32", c.max_row_weight);
    SpTables& t = x->spt;
    if (c.z > SP_MAXT) return fail(LDPC_ERR_UNSUPPORTED, "float decoder: Z=%d > %d", c.z, SP_MAXT);
    int G = std::max(1, std::min(32, 128 / c.z));
    if (const char* e = getenv("LDPC_SP_G")) G = std::max(1, std::min(32, atoi(e)));
    while (G > 1 && ((G * c.z + 31) / 32) * 32 > SP_MAXT) --G;
    fill_sp_tables(c, G, &t);
    x->sp_threads = ((G * c.z + 31) / 32) * 32;
    const int nstage = (t.n + 3) & ~3;
    const size_t base_smem = ((((size_t)G * t.stride + 3) & ~(size_t)3) + (size_t)G * nstage) * 4;
    const size_t r_smem = (size_t)t.E * x->sp_threads * 4;
    const bool rsmem = base_smem + r_smem <= 160 * 1024;
    const SpVariant* v = nullptr;
    for (const SpVariant& k : kSp)
        if (k.dmax == dmax && k.prod == prod && k.rsmem == rsmem) v = &k;
    x->sp_kernel = v->k;
    x->sp_smem = (int)(base_smem + (rsmem ? r_smem : 0));
    // up to 220 KB dynamic (B200: 227 KB per CTA, less the kernel's static shared memory)
    if (x->sp_smem > kSpMaxSmem) return fail(LDPC_ERR_UNSUPPORTED, "float decoder: %d B of shared memory", x->sp_smem);
    CUDA_TRY(allow_dynamic_smem((const void*)v->k, kSpMaxSmem));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)v->k, x->sp_threads, x->sp_smem));
    if (per_sm < 1) return fail(LDPC_ERR_UNSUPPORTED, "float decoder: launch does not fit an SM");
    x->sp_ctas = per_sm * x->sms;
    if (!rsmem) {
        CUDA_TRY(cudaMalloc(&x->d_sp_scratch, (size_t)x->sp_ctas * r_smem));
    }
    // decode_row's Max_row_simd (decode_functions.cpp:27-32) for a float build
    x->maxf = x->cfg.max_row_metric < 1e-6 ? (float)(1.0 - (double)x->cfg.max_row_metric) : x->cfg.max_row_metric;
    return LDPC_OK;
}

int launch_sp(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s) {
    if (!x->sp_kernel) return fail(LDPC_ERR_INVALID_ARG, "context was not created for a float decoder");
    if (a.n == 0) return LDPC_OK;
    SpJob job;
    memset(&job, 0, sizeof(job));
    job.llr = (const float*)a.llr;
    job.ncw = (long long)a.n;
    job.post_out = (float*)a.post;
    job.hard_out = a.hard;
    job.iters_out = a.iters;
    job.ref_bits = a.ref_bits;
    job.ref_period = a.ref_period > 0 ? a.ref_period : 1;
    job.bucket_size = a.bucket_size > 0 ? a.bucket_size : (long long)a.n;
    job.counters = a.counters;
    job.n_buckets = std::max(1, std::min(a.n_buckets, OMS_MAX_BUCKETS));
    job.num_par = x->code.num_par;
    job.max_iter = (int)x->cfg.max_iter;
    job.prod = x->cfg.variant == LDPC_F32_SP;
    job.beta = x->cfg.beta;
    job.maxv = x->maxf;
    job.r_scratch = x->d_sp_scratch;
    const long long want = ((long long)a.n + x->spt.G - 1) / x->spt.G;
    const int grid = (int)std::min<long long>(want, x->sp_ctas);
    x->sp_kernel<<<grid, x->sp_threads, x->sp_smem, s>>>(x->spt, job);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

}  // namespace ldpc
