// Host side of the int8 offset min-sum decoder over run-time code tables:
// code description, launch geometry, single-code launch.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.h"
#include "oms_rt.cuh"

namespace ldpc {

namespace {
struct RtVariant {
    int dmax;
    bool quirk, rsmem;
    rt_fn k;
};
#define RTV(D_) {D_, false, false, oms_rt_kernel<D_, false, false>}, {D_, false, true, oms_rt_kernel<D_, false, true>}, \
                {D_, true, false, oms_rt_kernel<D_, true, false>},   {D_, true, true, oms_rt_kernel<D_, true, true>}
const RtVariant kRt[] = {RTV(8), RTV(12), RTV(16), RTV(24), RTV(32)};
#undef RTV

}  // namespace

rt_fn rt_kernel_for(int dmax, bool quirk, bool rsmem) {
    for (const RtVariant& v : kRt)
        if (v.dmax == dmax && v.quirk == quirk && v.rsmem == rsmem) return v.k;
    return nullptr;
}

// posterior stride: n rounded so that stride mod 32 = ceil(32/G)
int rt_stride(int n, int G) {
    const int spread = (32 + G - 1) / G;
    return n + (((spread - n) % 32) + 32) % 32;
}

size_t rt_smem_bytes(int n, int G, int E, int threads, bool rsmem) {
    const size_t nstage = (size_t)((n + 15) & ~15);
    return (size_t)rt_code_bytes() + (((size_t)G * rt_stride(n, G) * 4 + 15) & ~(size_t)15) + 2 * (size_t)G * nstage +
           (rsmem ? (size_t)(E | 1) * threads * 4 : 0);   // odd per-thread stride
}

int rt_default_G(int z, int n) {
    const int cap = n <= 2048 ? 128 : 256;
    int G = 1;
    double best = 0.0;
    for (int g = 1; g <= 16 && g * z <= cap; ++g) {
        const double eff = (double)(g * z) / (((g * z + 31) / 32) * 32);
        if (eff >= best - 1e-9) {
            best = eff;
            G = g;
        }
    }
    return G;
}

int rt_dmax(int d) { return d <= 8 ? 8 : d <= 12 ? 12 : d <= 16 ? 16 : d <= 24 ? 24 : d <= 32 ? 32 : 0; }

int make_rt_code(const ldpc_code& c, int max_iter, uint32_t maxv2, const int* beta8, int beta8_all, int G, RtCode* out) {
    const int E = (int)c.row_cols.size();
    if (c.mrow > RT_MAX_L || E > RT_MAX_E)
        return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: %d layers / %d circulants exceed %d / %d", c.mrow, E, RT_MAX_L,
                    RT_MAX_E);
    if (c.z > RT_MAX_Z) return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: Z=%d > %d", c.z, RT_MAX_Z);
    if (!rt_dmax(c.max_row_weight)) return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: row weight %d > 32", c.max_row_weight);
    if (G < 1 || G > 16) return fail(LDPC_ERR_INVALID_ARG, "int8 decoder: %d codeword pairs per CTA", G);
    RtCode& r = *out;
    memset(&r, 0, sizeof(r));
    r.z = c.z;
    r.n = c.z * c.mcol;
    r.L = c.mrow;
    r.E = E;
    r.G = G;
    r.stride = rt_stride(r.n, G);
    r.kbits = c.z * (c.mcol - c.mrow);
    r.hard_words = (r.kbits + 31) / 32;
    r.num_par = c.num_par;
    r.max_iter = max_iter;
    r.maxv2 = maxv2;
    int e0 = 0;
    for (int l = 0; l < c.mrow; ++l) {
        const int b = beta8 ? beta8[l] : beta8_all;
        if (b < 0 || b > 127) return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: offset %d of layer %d outside 0..127", b, l);
        r.beta2[l] = half2_bits((float)b);
        r.quirk2[l] = b == 0 ? 0xd800d800u : 0u;
        r.rw[l] = (int16_t)c.row_weights[l];
        r.ebase[l] = (int16_t)e0;
        e0 += c.row_weights[l];
    }
    for (int e = 0; e < E; ++e) r.edge[e] = ((uint32_t)(c.row_cols[e] * c.z) << 9) | (uint32_t)c.row_shifts[e];
    return LDPC_OK;
}

int setup_oms_rt(ldpc_ctx* x) {
    const ldpc_code& c = x->code;
    const int E = (int)c.row_cols.size();
    const int n = c.z * c.mcol;
    const int dmax = rt_dmax(c.max_row_weight);
    if (!dmax) return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: row weight %d > 32", c.max_row_weight);
    if (c.z > kRtMaxThreads) return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: Z=%d > %d", c.z, kRtMaxThreads);
    bool quirk = x->layer_beta8.empty() && !x->tab_rows && x->beta0;
    for (int v : x->layer_beta8) quirk |= v == 0;
    for (int v : x->tab_beta8) quirk |= v == 0;
    const bool force_global = getenv("LDPC_OMS_RT_GLOBAL") != nullptr;
    // Codeword pairs per CTA (LDPC_OMS_G overrides): CTAs of at most 128
    // threads for codes of N <= 2048 (short barriers, several CTAs per SM),
    // 256 for longer ones, and of those the G whose G Z rows leave the fewest
    // of the CTA's lanes idle (the larger G on a tie; G = 1 when Z exceeds the
    // cap).  Measured over G = 1..16 on fourteen 802.11ad/ay, 802.11n,
    // 802.16e, G.hn and 5G NR codes this is the fastest shape or within 9 %
    // of it; the former ~256-thread default for every code lost up to 35 % on
    // the short ones, a 128-thread cap up to 41 % on 5G NR base graph 2.
    int G = rt_default_G(c.z, n);
    if (const char* e = getenv("LDPC_OMS_G")) G = std::max(1, std::min(16, atoi(e)));
    while (G > 1 && ((G * c.z + 31) / 32) * 32 > kRtMaxThreads) --G;
    while (G > 1 && rt_smem_bytes(n, G, E, 0, false) > (size_t)kRtMaxSmem) --G;
    const int threads = ((G * c.z + 31) / 32) * 32;
    bool rsmem = !force_global && rt_smem_bytes(n, G, E, threads, true) <= (size_t)kRtMaxSmem;
    const size_t smem = rt_smem_bytes(n, G, E, threads, rsmem);
    if (smem > (size_t)kRtMaxSmem)
        return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: N=%d needs %zu B of shared memory", n, smem);
    RtCode host;
    const int* table = x->layer_beta8.empty() ? nullptr : x->layer_beta8.data();
    int rc = make_rt_code(c, (int)x->cfg.max_iter, x->maxv2, table, (int)(int8_t)x->cfg.beta, G, &host);
    if (rc) return rc;
    if (x->tab_rows) {
        std::vector<uint16_t> h(x->tab_beta8.size());
        for (size_t i = 0; i < h.size(); ++i) h[i] = (uint16_t)half2_bits((float)x->tab_beta8[i]);
        CUDA_TRY(cudaMalloc(&x->d_beta_tab, h.size() * sizeof(uint16_t)));
        CUDA_TRY(cudaMemcpy(x->d_beta_tab, h.data(), h.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
        host.beta_tab = x->d_beta_tab;
        host.tab_rows = x->tab_rows;
    }
    rt_fn k = rt_kernel_for(dmax, quirk, rsmem);
    CUDA_TRY(allow_dynamic_smem((const void*)k, kRtMaxSmem));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k, threads, smem));
    if (per_sm < 1) return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: %d threads x %zu B do not fit an SM", threads, smem);
    x->rt_ctas = per_sm * x->sms;
    CUDA_TRY(cudaMalloc(&x->d_rt_code, sizeof(RtCode)));
    CUDA_TRY(cudaMemcpy(x->d_rt_code, &host, sizeof(RtCode), cudaMemcpyHostToDevice));
    if (!rsmem) {
        x->rt_words_per_cta = (long long)E * threads;
        CUDA_TRY(cudaMalloc(&x->d_rt_scratch, (size_t)x->rt_ctas * x->rt_words_per_cta * 4));
    }
    x->rt_kernel = k;
    x->rt_threads = threads;
    x->rt_smem = (int)smem;
    x->rt_G = G;
    x->oms_rt = true;
    return LDPC_OK;
}

int launch_oms_rt(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s) {
    if (a.n == 0) return LDPC_OK;
    RtLaunch lp;
    memset(&lp, 0, sizeof(lp));
    lp.codes = x->d_rt_code;
    RtJob& j = lp.job0;
    j.llr = (const int8_t*)a.llr;
    j.ncw = (long long)a.n;
    j.post_out = (int8_t*)a.post;
    j.hard_out = a.hard;
    j.iters_out = a.iters;
    j.ref_bits = a.ref_bits;
    j.ref_period = a.ref_period > 0 ? a.ref_period : 1;
    j.bucket_size = a.bucket_size > 0 ? a.bucket_size : (long long)a.n;
    j.counters = a.counters;
    j.n_buckets = std::max(1, std::min(a.n_buckets, OMS_MAX_BUCKETS));
    j.code = 0;
    lp.r_scratch = x->d_rt_scratch;
    lp.r_words_per_cta = x->rt_words_per_cta;
    const long long slots = 2LL * x->rt_G;
    const long long want = ((long long)a.n + slots - 1) / slots;
    const int grid = (int)std::min<long long>(want, x->rt_ctas);
    x->rt_kernel<<<grid, x->rt_threads, x->rt_smem, s>>>(lp);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

}  // namespace ldpc
