// Host side of the float and double decoders (sum-product, offset min-sum).
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
    sp64_fn k64;
};
#define SPV(D_, P_, R_) {D_, P_, R_, sp_f32_kernel<D_, P_, R_, SP_MAXT>, sp_f64_kernel<D_, P_, R_, SP_MAXT>}
const SpVariant kSp[] = {
    SPV(8, true, true),  SPV(8, true, false),  SPV(8, false, true),  SPV(8, false, false),
    SPV(16, true, true), SPV(16, true, false), SPV(16, false, true), SPV(16, false, false),
    SPV(32, true, true), SPV(32, true, false), SPV(32, false, true), SPV(32, false, false),
};
#undef SPV

bool is_f64(int variant) { return variant == LDPC_F64_SP || variant == LDPC_F64_OMS; }
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
    const bool dbl = is_f64(x->cfg.variant);
    const bool prod = x->cfg.variant == LDPC_F32_SP || x->cfg.variant == LDPC_F64_SP;
    const size_t es = dbl ? 8 : 4;              // bytes per element
    const int V = 16 / (int)es;                 // elements per 16 bytes
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
    // posteriors + staging of G codewords; fewer codewords per CTA while that
    // exceeds the shared memory, then no staging buffer
    const int nstage = (c.z * c.mcol + V - 1) & ~(V - 1);
    auto base_bytes = [&](int g, bool stage) {
        fill_sp_tables(c, g, &t);
        return ((((size_t)g * t.stride + V - 1) & ~(size_t)(V - 1)) + (stage ? (size_t)g * nstage : 0)) * es;
    };
    while (G > 1 && base_bytes(G, true) > (size_t)kSpMaxSmem) --G;
    const bool nostage = base_bytes(G, true) > (size_t)kSpMaxSmem;
    const size_t base_smem = base_bytes(G, !nostage);   // leaves t filled for G
    t.nostage = nostage ? 1 : 0;
    x->sp_threads = ((G * c.z + 31) / 32) * 32;
    // messages: shared memory holds E | 1 per thread (odd stride), the global
    // scratch E per thread
    const size_t r_smem = (size_t)(t.E | 1) * x->sp_threads * es;
    const size_t r_glob = (size_t)t.E * x->sp_threads * es;
    // sum-product: messages in shared memory unless messages in global
    // scratch (L2) give at least 1.5 times the CTAs per SM -- its tanh/atanh
    // chains are latency-bound, so resident warps count for more than
    // message latency, but one CTA more out of five does not pay for the L2
    // round trips (802.11ad float: 6 vs 5 CTAs is 5 % slower).  Min-sum,
    // light on arithmetic, keeps them in shared memory whenever they fit.
    auto find = [&](bool rs) {
        const SpVariant* f = nullptr;
        for (const SpVariant& k : kSp)
            if (k.dmax == dmax && k.prod == prod && k.rsmem == rs) f = &k;
        return f;
    };
    auto ctas_per_sm = [&](const SpVariant* k, size_t bytes, int* out) -> cudaError_t {
        const void* fn = dbl ? (const void*)k->k64 : (const void*)k->k;
        cudaError_t e = allow_dynamic_smem(fn, kSpMaxSmem);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, fn, x->sp_threads, bytes);
        return e;
    };
    // tuning: LDPC_SP_RGLOBAL forces global messages, LDPC_SP_RSMEM shared
    // ones where they fit
    bool rsmem = false;
    if (base_smem + r_smem <= 160 * 1024 && !getenv("LDPC_SP_RGLOBAL")) {
        int per_s = 0, per_g = 0;
        CUDA_TRY(ctas_per_sm(find(true), base_smem + r_smem, &per_s));
        CUDA_TRY(ctas_per_sm(find(false), base_smem, &per_g));
        rsmem = !prod || 2 * per_g < 3 * per_s || getenv("LDPC_SP_RSMEM");
    }
    const SpVariant* v = find(rsmem);
    x->sp_kernel = dbl ? nullptr : v->k;
    x->sp64_kernel = dbl ? v->k64 : nullptr;
    const void* kfn = dbl ? (const void*)v->k64 : (const void*)v->k;
    x->sp_smem = (int)(base_smem + (rsmem ? r_smem : 0));
    // up to 220 KB dynamic (B200: 227 KB per CTA, less the kernel's static shared memory)
    if (x->sp_smem > kSpMaxSmem)
        return fail(LDPC_ERR_UNSUPPORTED, "%s decoder: %d B of shared memory", dbl ? "double" : "float", x->sp_smem);
    CUDA_TRY(allow_dynamic_smem(kfn, kSpMaxSmem));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, x->sp_threads, x->sp_smem));
    if (per_sm < 1) return fail(LDPC_ERR_UNSUPPORTED, "float decoder: launch does not fit an SM");
    x->sp_ctas = per_sm * x->sms;
    if (!rsmem) {
        CUDA_TRY(cudaMalloc(&x->d_sp_scratch, (size_t)x->sp_ctas * r_glob));
    }
    // decode_row's Max_row_simd (decode_functions.cpp:27-32): 1 - (CTYPE)max_row_metric
    // below 1e-6 (sum-product), else max_row_metric, in the build's element type
    const double mrm = (double)x->cfg.max_row_metric;
    x->maxf = x->cfg.max_row_metric < 1e-6 ? (float)(1.0 - mrm) : x->cfg.max_row_metric;
    x->maxd = x->cfg.max_row_metric < 1e-6 ? 1.0 - mrm : mrm;
    return LDPC_OK;
}

namespace {
template <class T>
SpJobT<T> sp_job(const ldpc_ctx* x, const DecodeArgs& a, T maxv) {
    SpJobT<T> job;
    memset(&job, 0, sizeof(job));
    job.llr = (const T*)a.llr;
    job.ncw = (long long)a.n;
    job.post_out = (T*)a.post;
    job.hard_out = a.hard;
    job.iters_out = a.iters;
    job.ref_bits = a.ref_bits;
    job.ref_period = a.ref_period > 0 ? a.ref_period : 1;
    job.bucket_size = a.bucket_size > 0 ? a.bucket_size : (long long)a.n;
    job.counters = a.counters;
    job.n_buckets = std::max(1, std::min(a.n_buckets, OMS_MAX_BUCKETS));
    job.num_par = x->code.num_par;
    job.max_iter = (int)x->cfg.max_iter;
    job.prod = x->cfg.variant == LDPC_F32_SP || x->cfg.variant == LDPC_F64_SP;
    job.beta = (T)x->cfg.beta;
    job.maxv = maxv;
    job.r_scratch = (T*)x->d_sp_scratch;
    return job;
}
}  // namespace

int launch_sp(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s) {
    if (!x->sp_kernel && !x->sp64_kernel) return fail(LDPC_ERR_INVALID_ARG, "context was not created for a float decoder");
    if (a.n == 0) return LDPC_OK;
    const long long want = ((long long)a.n + x->spt.G - 1) / x->spt.G;
    const int grid = (int)std::min<long long>(want, x->sp_ctas);
    if (x->sp64_kernel)
        x->sp64_kernel<<<grid, x->sp_threads, x->sp_smem, s>>>(x->spt, sp_job<double>(x, a, x->maxd));
    else
        x->sp_kernel<<<grid, x->sp_threads, x->sp_smem, s>>>(x->spt, sp_job<float>(x, a, x->maxf));
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

}  // namespace ldpc
