// Batched decoding: several codes (and Z sizes) in one persistent launch of
// the run-time-table int8 kernel, plans with CUDA-graph replay, and the
// launch-shape autotuner.  An int8 plan whose codes would run at different
// occupancies (shared memory, message placement, row-weight bucket) is split
// into one persistent launch per class; its graph holds one kernel node per
// class with no dependencies between them, so the classes overlap.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "internal.h"
#include "sp_batch.cuh"

using ldpc::fail;

struct ldpc_batch {
    int device = 0, sms = 0;
    int variant = LDPC_INT8_OMS;             // every code of a batch runs the same decoder
    std::vector<float> maxf;                 // float batches: decode_row's Max_val per code
    std::vector<ldpc_code> codes;
    std::vector<ldpc_cfg> cfgs;
    std::vector<std::vector<int>> beta8;     // per code, per layer
    std::vector<std::vector<int>> tab8;      // per code: int8 offset table [rows][layer], or empty
    std::vector<int> tab_rows;
    std::vector<uint32_t> maxv2;
    int tuned_threads = 0, tuned_cpc = 0;    // one launch shape for all codes (float, or one class)
    std::vector<int> code_threads, code_cpc;  // int8 per-class tuning, per code (0 = untuned)
};

struct ldpc_batch_plan {
    int device = 0;
    bool is_float = false;
    ldpc::RtLaunch lp;                       // int8 batches
    ldpc::rt_fn k = nullptr;
    ldpc::SpBatchLaunch slp;                 // float batches
    void* kf = nullptr;
    int threads = 0, smem = 0, grid = 0, n_chunks = 0;
    void* d_codes = nullptr;
    void* d_jobs = nullptr;
    ldpc::RtChunk* d_chunks = nullptr;
    void* d_scratch = nullptr;
    uint16_t* d_tabs = nullptr;              // offset tables of the plan's codes (half bits)
    unsigned int* d_claim = nullptr;        // chunk-claim counter, zeroed before each launch
    cudaStream_t own = nullptr;              // graph capture and replay stream
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<ldpc_batch_plan*> parts;      // per-class launches (owned); empty: this plan is one launch
};

namespace {

constexpr int kTunedWidths[] = {128, 192, 256, 320, 384, 448, 512};

typedef void (*spb_fn)(const ldpc::SpBatchLaunch);
struct SpbVariant {
    int dmax;
    bool prod, rsmem;
    spb_fn k;
};
#define SPB(D_, P_, R_) {D_, P_, R_, ldpc::sp_batch_kernel<D_, P_, R_>}
const SpbVariant kSpb[] = {SPB(8, true, true),   SPB(8, true, false),   SPB(8, false, true),   SPB(8, false, false),
                           SPB(16, true, true),  SPB(16, true, false),  SPB(16, false, true),  SPB(16, false, false),
                           SPB(32, true, true),  SPB(32, true, false),  SPB(32, false, true),  SPB(32, false, false)};
#undef SPB

cudaError_t launch_plan_kernel(ldpc_batch_plan* p, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(p->d_claim, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    if (p->is_float) ((spb_fn)p->kf)<<<p->grid, p->threads, p->smem, s>>>(p->slp);
    else p->k<<<p->grid, p->threads, p->smem, s>>>(p->lp);
    return cudaGetLastError();
}

// Chunks of about equal work (codewords x edges per codeword) so that the
// strided chunk-to-CTA assignment balances the CTAs.
void make_chunks(const std::vector<long long>& ncw, const std::vector<long long>& cost_per_cw,
                 const std::vector<int>& min_chunk, long long target_chunks, std::vector<ldpc::RtChunk>& out) {
    double total = 0;
    for (size_t j = 0; j < ncw.size(); ++j) total += (double)ncw[j] * (double)cost_per_cw[j];
    const double per_chunk = std::max(1.0, total / (double)std::max(1LL, target_chunks));
    for (size_t j = 0; j < ncw.size(); ++j) {
        const long long n = ncw[j];
        if (n == 0) continue;
        long long m = (long long)std::llround((double)n * (double)cost_per_cw[j] / per_chunk);
        m = std::max(1LL, std::min(m, std::max(1LL, n / min_chunk[j])));
        for (long long i = 0; i < m; ++i) {
            ldpc::RtChunk c;
            c.job = (int)j;
            c.pad = 0;
            c.lo = n * i / m;
            c.hi = n * (i + 1) / m;
            out.push_back(c);
        }
    }
}

int check_job(const ldpc_batch* b, const ldpc_batch_job& j, int idx) {
    if (j.code < 0 || j.code >= (int)b->codes.size()) return fail(LDPC_ERR_INVALID_ARG, "job %d: code %d of %zu", idx, j.code, b->codes.size());
    if (j.n && !j.llr) return fail(LDPC_ERR_INVALID_ARG, "job %d: llr is NULL", idx);
    if (j.n > (size_t)1 << 40) return fail(LDPC_ERR_INVALID_ARG, "job %d: n=%zu too large", idx, j.n);
    if (j.counters && (!j.data_bits || j.ref_period == 0 || j.n_buckets < 1 || j.n_buckets > ldpc::OMS_MAX_BUCKETS))
        return fail(LDPC_ERR_INVALID_ARG, "job %d: counting needs data_bits, ref_period > 0 and 1..%d buckets", idx,
                    ldpc::OMS_MAX_BUCKETS);
    return LDPC_OK;
}

void release(ldpc_batch_plan* p);

void destroy_plan(ldpc_batch_plan* p) {
    if (p) {
        cudaSetDevice(p->device);
        release(p);
        delete p;
    }
}

void release(ldpc_batch_plan* p) {
    for (ldpc_batch_plan* q : p->parts) destroy_plan(q);
    p->parts.clear();
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->ev_in) cudaEventDestroy(p->ev_in);
    if (p->ev_out) cudaEventDestroy(p->ev_out);
    if (p->own) cudaStreamDestroy(p->own);
    cudaFree(p->d_codes);
    cudaFree(p->d_jobs);
    cudaFree(p->d_chunks);
    cudaFree(p->d_scratch);
    cudaFree(p->d_tabs);
    cudaFree(p->d_claim);
}

struct PlanDel {
    void operator()(ldpc_batch_plan* p) const { destroy_plan(p); }
};

int float_plan(ldpc_batch* b, const ldpc_batch_job* jobs, int n_jobs, int threads, int cpc, ldpc_batch_plan** out) {
    const int nc = (int)b->codes.size();
    const bool prod = b->variant == LDPC_F32_SP;
    std::vector<char> used(nc, 0);
    for (int i = 0; i < n_jobs; ++i) used[jobs[i].code] = 1;
    std::vector<int> G(nc, 1);
    std::vector<size_t> base(nc, 0);
    int dmax = 8, maxE = 0;
    bool rsmem = !getenv("LDPC_SP_RGLOBAL");
    for (int c = 0; c < nc; ++c) {
        if (!used[c]) continue;
        const ldpc_code& cd = b->codes[c];
        const int n = cd.z * cd.mcol, E = (int)cd.row_cols.size();
        auto bytes = [&](int g) {
            ldpc::SpTables t;
            ldpc::fill_sp_tables(cd, g, &t);
            return (size_t)ldpc::sp_code_bytes() + (((size_t)g * t.stride + 3) & ~(size_t)3) * 4 + (size_t)g * ((n + 3) & ~3) * 4;
        };
        G[c] = std::max(1, std::min(32, threads / cd.z));
        while (G[c] > 1 && bytes(G[c]) > (size_t)ldpc::kSpMaxSmem) --G[c];
        base[c] = bytes(G[c]);
        if (base[c] > (size_t)ldpc::kSpMaxSmem)
            return fail(LDPC_ERR_UNSUPPORTED, "batch plan: code %d (N=%d) does not fit shared memory", c, n);
        if (base[c] + (size_t)(E | 1) * threads * 4 > (size_t)ldpc::kSpMaxSmem) rsmem = false;   // odd per-thread stride
        dmax = std::max(dmax, cd.max_row_weight <= 8 ? 8 : cd.max_row_weight <= 16 ? 16 : 32);
        maxE = std::max(maxE, E);
    }
    auto find = [&](bool rs) {
        spb_fn f = nullptr;
        for (const SpbVariant& v : kSpb)
            if (v.dmax == dmax && v.prod == prod && v.rsmem == rs) f = v.k;
        return f;
    };
    auto smem_of = [&](bool rs) {
        size_t m = 0;
        for (int c = 0; c < nc; ++c)
            if (used[c]) m = std::max(m, base[c] + (rs ? (size_t)((int)b->codes[c].row_cols.size() | 1) * threads * 4 : 0));
        return m;
    };
    if (rsmem && prod) {
        // as for a single code: sum-product keeps shared-memory messages
        // unless global (L2) messages give at least 1.5 times the CTAs per SM
        int per_s = 0, per_g = 0;
        CUDA_TRY(ldpc::allow_dynamic_smem((const void*)find(true), ldpc::kSpMaxSmem));
        CUDA_TRY(ldpc::allow_dynamic_smem((const void*)find(false), ldpc::kSpMaxSmem));
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_s, (const void*)find(true), threads, smem_of(true)));
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_g, (const void*)find(false), threads, smem_of(false)));
        rsmem = 2 * per_g < 3 * per_s;
    }
    const size_t smem = smem_of(rsmem);
    spb_fn k = find(rsmem);
    std::unique_ptr<ldpc_batch_plan, PlanDel> p(new ldpc_batch_plan);
    p->device = b->device;
    p->is_float = true;
    p->kf = (void*)k;
    p->threads = threads;
    p->smem = (int)smem;
    CUDA_TRY(ldpc::allow_dynamic_smem((const void*)k, ldpc::kSpMaxSmem));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k, threads, smem));
    if (per_sm < 1) return fail(LDPC_ERR_UNSUPPORTED, "batch plan: %d threads x %zu B do not fit an SM", threads, smem);
    const long long ctas = (long long)per_sm * b->sms;
    std::vector<ldpc::SpCode> hc(nc);
    for (int c = 0; c < nc; ++c) {
        memset(&hc[c], 0, sizeof(hc[c]));
        ldpc::fill_sp_tables(b->codes[c], G[c], &hc[c].t);
        hc[c].max_iter = (int)b->cfgs[c].max_iter;
        hc[c].num_par = b->codes[c].num_par;
        hc[c].beta = b->cfgs[c].beta;
        hc[c].maxv = b->maxf[c];
    }
    std::vector<ldpc::SpBatchJob> hj(n_jobs);
    std::vector<long long> ncw(n_jobs), cost(n_jobs);
    std::vector<int> minc(n_jobs);
    for (int i = 0; i < n_jobs; ++i) {
        const ldpc_batch_job& s = jobs[i];
        ldpc::SpBatchJob& j = hj[i];
        memset(&j, 0, sizeof(j));
        j.llr = (const float*)s.llr;
        j.ncw = (long long)s.n;
        j.post_out = (float*)s.post_out;
        j.hard_out = s.hard_out;
        j.iters_out = s.iters_out;
        j.ref_bits = s.data_bits;
        j.ref_period = s.ref_period > 0 ? (long long)s.ref_period : 1;
        j.bucket_size = s.bucket_size > 0 ? (long long)s.bucket_size : std::max(1LL, (long long)s.n);
        j.counters = s.counters;
        j.n_buckets = std::max(1, std::min(s.n_buckets, ldpc::OMS_MAX_BUCKETS));
        j.code = s.code;
        const ldpc_code& cd = b->codes[s.code];
        ncw[i] = j.ncw;
        cost[i] = (long long)cd.row_cols.size() * cd.z;
        minc[i] = 4 * G[s.code];
    }
    std::vector<ldpc::RtChunk> chunks;
    make_chunks(ncw, cost, minc, ctas * cpc, chunks);
    const int n_chunks = (int)chunks.size();
    p->grid = (int)std::max(1LL, std::min<long long>(ctas, n_chunks));
    CUDA_TRY(cudaMalloc(&p->d_codes, sizeof(ldpc::SpCode) * nc));
    CUDA_TRY(cudaMemcpy(p->d_codes, hc.data(), sizeof(ldpc::SpCode) * nc, cudaMemcpyHostToDevice));
    if (n_jobs) {
        CUDA_TRY(cudaMalloc(&p->d_jobs, sizeof(ldpc::SpBatchJob) * n_jobs));
        CUDA_TRY(cudaMemcpy(p->d_jobs, hj.data(), sizeof(ldpc::SpBatchJob) * n_jobs, cudaMemcpyHostToDevice));
    }
    if (n_chunks) {
        CUDA_TRY(cudaMalloc(&p->d_chunks, sizeof(ldpc::RtChunk) * n_chunks));
        CUDA_TRY(cudaMemcpy(p->d_chunks, chunks.data(), sizeof(ldpc::RtChunk) * n_chunks, cudaMemcpyHostToDevice));
    }
    long long words = 0;
    if (!rsmem) {
        words = (long long)maxE * threads;
        CUDA_TRY(cudaMalloc(&p->d_scratch, (size_t)p->grid * words * 4));
    }
    memset(&p->slp, 0, sizeof(p->slp));
    p->slp.codes = (const ldpc::SpCode*)p->d_codes;
    p->slp.jobs = (const ldpc::SpBatchJob*)p->d_jobs;
    p->slp.chunks = p->d_chunks;
    p->slp.n_chunks = p->d_jobs ? n_chunks : 0;
    p->slp.r_scratch = (float*)p->d_scratch;
    p->slp.r_words_per_cta = words;
    CUDA_TRY(cudaMalloc(&p->d_claim, sizeof(unsigned int)));
    p->slp.claim = p->d_claim;
    p->n_chunks = p->slp.n_chunks;
    *out = p.release();
    return LDPC_OK;
}

// One persistent launch of the run-time-table int8 kernel over the jobs; its
// kernel variant, shared memory and message placement come from the codes
// the jobs use.
int int8_plan(ldpc_batch* b, const ldpc_batch_job* jobs, int n_jobs, int threads, int cpc, ldpc_batch_plan** out) {
    const int nc = (int)b->codes.size();
    std::vector<char> used(nc, 0);
    for (int i = 0; i < n_jobs; ++i) used[jobs[i].code] = 1;
    std::vector<int> G(nc, 1);
    int dmax = 8, maxE = 0;
    bool quirk = false, rsmem = true;
    for (int c = 0; c < nc; ++c) {
        if (!used[c]) continue;
        const ldpc_code& cd = b->codes[c];
        const int n = cd.z * cd.mcol, E = (int)cd.row_cols.size();
        G[c] = std::max(1, std::min(16, threads / cd.z));
        while (G[c] > 1 && ldpc::rt_smem_bytes(n, G[c], E, 0, false) > (size_t)ldpc::kRtMaxSmem) --G[c];
        if (ldpc::rt_smem_bytes(n, G[c], E, 0, false) > (size_t)ldpc::kRtMaxSmem)
            return fail(LDPC_ERR_UNSUPPORTED, "batch plan: code %d (N=%d) does not fit shared memory", c, n);
        if (ldpc::rt_smem_bytes(n, G[c], E, threads, true) > (size_t)ldpc::kRtMaxSmem) rsmem = false;
        dmax = std::max(dmax, ldpc::rt_dmax(cd.max_row_weight));
        maxE = std::max(maxE, E);
        for (int v : b->beta8[c]) quirk |= v == 0;
        for (int v : b->tab8[c]) quirk |= v == 0;
    }
    size_t smem = 0;
    for (int c = 0; c < nc; ++c) {
        if (!used[c]) continue;
        const ldpc_code& cd = b->codes[c];
        smem = std::max(smem, ldpc::rt_smem_bytes(cd.z * cd.mcol, G[c], (int)cd.row_cols.size(), threads, rsmem));
    }
    std::unique_ptr<ldpc_batch_plan, PlanDel> p(new ldpc_batch_plan);
    p->device = b->device;
    p->k = ldpc::rt_kernel_for(dmax, quirk, rsmem);
    p->threads = threads;
    p->smem = (int)smem;
    CUDA_TRY(ldpc::allow_dynamic_smem((const void*)p->k, ldpc::kRtMaxSmem));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)p->k, threads, smem));
    if (per_sm < 1) return fail(LDPC_ERR_UNSUPPORTED, "batch plan: %d threads x %zu B do not fit an SM", threads, smem);
    const long long ctas = (long long)per_sm * b->sms;

    std::vector<ldpc::RtCode> hc(nc);
    for (int c = 0; c < nc; ++c) {
        const ldpc_code& cd = b->codes[c];
        if (int rc = ldpc::make_rt_code(cd, (int)b->cfgs[c].max_iter, b->maxv2[c], b->beta8[c].data(), 0, G[c], &hc[c]))
            return rc;
    }
    // offset tables of the used codes, one device buffer
    std::vector<uint16_t> tabs;
    std::vector<size_t> tab_at(nc, 0);
    for (int c = 0; c < nc; ++c) {
        if (!used[c] || b->tab8[c].empty()) continue;
        tab_at[c] = tabs.size();
        for (int v : b->tab8[c]) tabs.push_back((uint16_t)ldpc::half2_bits((float)v));
    }
    if (!tabs.empty()) {
        CUDA_TRY(cudaMalloc(&p->d_tabs, tabs.size() * sizeof(uint16_t)));
        CUDA_TRY(cudaMemcpy(p->d_tabs, tabs.data(), tabs.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
        for (int c = 0; c < nc; ++c) {
            if (!used[c] || b->tab8[c].empty()) continue;
            hc[c].beta_tab = p->d_tabs + tab_at[c];
            hc[c].tab_rows = b->tab_rows[c];
        }
    }
    std::vector<ldpc::RtJob> hj(n_jobs);
    std::vector<long long> cost(n_jobs);
    std::vector<int> minc(n_jobs);
    for (int i = 0; i < n_jobs; ++i) {
        const ldpc_batch_job& s = jobs[i];
        ldpc::RtJob& j = hj[i];
        memset(&j, 0, sizeof(j));
        j.llr = (const int8_t*)s.llr;
        j.ncw = (long long)s.n;
        j.post_out = (int8_t*)s.post_out;
        j.hard_out = s.hard_out;
        j.iters_out = s.iters_out;
        j.ref_bits = s.data_bits;
        j.ref_period = s.ref_period > 0 ? (long long)s.ref_period : 1;
        j.bucket_size = s.bucket_size > 0 ? (long long)s.bucket_size : std::max(1LL, (long long)s.n);
        j.counters = s.counters;
        j.n_buckets = std::max(1, std::min(s.n_buckets, ldpc::OMS_MAX_BUCKETS));
        j.code = s.code;
        const ldpc_code& cd = b->codes[s.code];
        cost[i] = (long long)cd.row_cols.size() * cd.z;
        minc[i] = 8 * G[s.code];     // a chunk keeps its 2G slots busy for a while
    }
    std::vector<ldpc::RtChunk> chunks;
    std::vector<long long> ncw(n_jobs);
    for (int i = 0; i < n_jobs; ++i) ncw[i] = hj[i].ncw;
    make_chunks(ncw, cost, minc, ctas * cpc, chunks);
    const int n_chunks = (int)chunks.size();
    p->grid = (int)std::max(1LL, std::min<long long>(ctas, n_chunks));
    CUDA_TRY(cudaMalloc(&p->d_codes, sizeof(ldpc::RtCode) * nc));
    CUDA_TRY(cudaMemcpy(p->d_codes, hc.data(), sizeof(ldpc::RtCode) * nc, cudaMemcpyHostToDevice));
    if (n_jobs) {
        CUDA_TRY(cudaMalloc(&p->d_jobs, sizeof(ldpc::RtJob) * n_jobs));
        CUDA_TRY(cudaMemcpy(p->d_jobs, hj.data(), sizeof(ldpc::RtJob) * n_jobs, cudaMemcpyHostToDevice));
    }
    if (n_chunks) {
        CUDA_TRY(cudaMalloc(&p->d_chunks, sizeof(ldpc::RtChunk) * n_chunks));
        CUDA_TRY(cudaMemcpy(p->d_chunks, chunks.data(), sizeof(ldpc::RtChunk) * n_chunks, cudaMemcpyHostToDevice));
    }
    long long words = 0;
    if (!rsmem) {
        words = (long long)maxE * threads;
        CUDA_TRY(cudaMalloc(&p->d_scratch, (size_t)p->grid * words * 4));
    }
    memset(&p->lp, 0, sizeof(p->lp));
    p->lp.codes = (const ldpc::RtCode*)p->d_codes;
    p->lp.jobs = (const ldpc::RtJob*)p->d_jobs;
    p->lp.chunks = p->d_chunks;
    p->lp.n_chunks = n_chunks;
    p->lp.r_scratch = (uint32_t*)p->d_scratch;
    p->lp.r_words_per_cta = words;
    CUDA_TRY(cudaMalloc(&p->d_claim, sizeof(unsigned int)));
    p->lp.claim = p->d_claim;
    if (!p->d_jobs) p->lp.n_chunks = 0;
    p->n_chunks = p->lp.n_chunks;
    *out = p.release();
    return LDPC_OK;
}

// Class of a code decoded alone at `threads`.  int8: kernel variant,
// message placement and CTAs per SM.  Float: the width and the row-weight
// bucket (the float kernel picks its message placement per launch).
struct PlanClass {
    int dmax = 0, quirk = 0, rsmem = 0, per_sm = 0, threads = 0;
    bool operator==(const PlanClass& o) const {
        return dmax == o.dmax && quirk == o.quirk && rsmem == o.rsmem && per_sm == o.per_sm && threads == o.threads;
    }
};

int int8_class(const ldpc_batch* b, int c, int threads, PlanClass* out) {
    const ldpc_code& cd = b->codes[c];
    const int n = cd.z * cd.mcol, E = (int)cd.row_cols.size();
    int G = std::max(1, std::min(16, threads / cd.z));
    while (G > 1 && ldpc::rt_smem_bytes(n, G, E, 0, false) > (size_t)ldpc::kRtMaxSmem) --G;
    const bool rsmem = ldpc::rt_smem_bytes(n, G, E, threads, true) <= (size_t)ldpc::kRtMaxSmem;
    bool quirk = false;
    for (int v : b->beta8[c]) quirk |= v == 0;
    for (int v : b->tab8[c]) quirk |= v == 0;
    const int dmax = ldpc::rt_dmax(cd.max_row_weight);
    ldpc::rt_fn k = ldpc::rt_kernel_for(dmax, quirk, rsmem);
    CUDA_TRY(ldpc::allow_dynamic_smem((const void*)k, ldpc::kRtMaxSmem));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k, threads,
                                                           ldpc::rt_smem_bytes(n, G, E, threads, rsmem)));
    out->dmax = dmax;
    out->quirk = quirk;
    out->rsmem = rsmem;
    out->per_sm = per_sm;
    out->threads = threads;
    return LDPC_OK;
}

// A code's own CTA width, the single-code context's: int8 G pairs of Z rows
// (rt_default_G: at most 128 threads, 256 for N > 2048, fewest idle lanes),
// float G = 128 / Z codewords per CTA; G*Z rounded to 32.
int default_width(const ldpc_batch* b, int c) {
    const int z = b->codes[c].z;
    if (b->variant == LDPC_INT8_OMS)
        return ((ldpc::rt_default_G(z, z * b->codes[c].mcol) * z + 31) / 32) * 32;
    const int G = std::max(1, std::min(32, 128 / z));
    return std::min(ldpc::kRtMaxThreads, ((G * z + 31) / 32) * 32);
}

// Class index of every code used by the jobs (code_cls[c], -1 if unused)
// and each class's width; returns the number of classes.  Widths: `threads`
// when explicit, else each code's own width.
int plan_classes(ldpc_batch* b, const ldpc_batch_job* jobs, int n_jobs, bool explicit_threads, int threads,
                 std::vector<int>& code_cls, std::vector<int>& cls_threads, int* n_cls) {
    const int nc = (int)b->codes.size();
    std::vector<PlanClass> cls;
    code_cls.assign(nc, -1);
    cls_threads.clear();
    for (int i = 0; i < n_jobs; ++i) {
        const int c = jobs[i].code;
        if (code_cls[c] >= 0) continue;
        PlanClass k;
        const int t = explicit_threads ? threads : default_width(b, c);
        if (b->variant == LDPC_INT8_OMS) {
            if (int rc = int8_class(b, c, t, &k)) return rc;
        } else {
            const int w = b->codes[c].max_row_weight;
            k.dmax = w <= 8 ? 8 : w <= 16 ? 16 : 32;
            k.threads = t;
        }
        int idx = -1;
        for (size_t j = 0; j < cls.size(); ++j)
            if (cls[j] == k) idx = (int)j;
        if (idx < 0) {
            idx = (int)cls.size();
            cls.push_back(k);
            cls_threads.push_back(t);
        }
        code_cls[c] = idx;
    }
    *n_cls = (int)cls.size();
    return LDPC_OK;
}

// The jobs of class k, and their largest Z.
std::vector<ldpc_batch_job> class_jobs(const ldpc_batch* b, const ldpc_batch_job* jobs, int n_jobs,
                                       const std::vector<int>& code_cls, int k, int* maxz) {
    std::vector<ldpc_batch_job> sub;
    *maxz = 0;
    for (int i = 0; i < n_jobs; ++i)
        if (code_cls[jobs[i].code] == k) {
            sub.push_back(jobs[i]);
            *maxz = std::max(*maxz, b->codes[jobs[i].code].z);
        }
    return sub;
}

int one_plan(ldpc_batch* b, const ldpc_batch_job* jobs, int n_jobs, int threads, int cpc, ldpc_batch_plan** out) {
    return b->variant == LDPC_INT8_OMS ? int8_plan(b, jobs, n_jobs, threads, cpc, out)
                                       : float_plan(b, jobs, n_jobs, threads, cpc, out);
}

// The jobs grouped by the class of their code; one launch per class (a
// single launch when there is one class, or when LDPC_BATCH_ONE_LAUNCH is
// set).  threads: the caller's width, applied to every class when explicit;
// otherwise each class takes its tuned shape (ldpc_batch_autotune) or its
// codes' own width and `cpc`.
int plans_by_class(ldpc_batch* b, const ldpc_batch_job* jobs, int n_jobs, bool explicit_threads, int threads,
                   int cpc, ldpc_batch_plan** out) {
    if (getenv("LDPC_BATCH_ONE_LAUNCH") || n_jobs < 2) return one_plan(b, jobs, n_jobs, threads, cpc, out);
    std::vector<int> code_cls, cls_threads;
    int n_cls = 0;
    if (int rc = plan_classes(b, jobs, n_jobs, explicit_threads, threads, code_cls, cls_threads, &n_cls)) return rc;
    if (n_cls < 2) {
        if (!explicit_threads && n_cls == 1) threads = cls_threads[0];
        return one_plan(b, jobs, n_jobs, threads, cpc, out);
    }
    std::unique_ptr<ldpc_batch_plan, PlanDel> p(new ldpc_batch_plan);
    p->device = b->device;
    for (int k = 0; k < n_cls; ++k) {
        int maxz = 0;
        std::vector<ldpc_batch_job> sub = class_jobs(b, jobs, n_jobs, code_cls, k, &maxz);
        int t = explicit_threads ? threads : cls_threads[k];
        int c = cpc;
        if (!explicit_threads && !b->code_threads.empty() && b->code_threads[sub[0].code] >= maxz) {
            t = b->code_threads[sub[0].code];
            c = b->code_cpc[sub[0].code];
        }
        ldpc_batch_plan* part = nullptr;
        if (int rc = one_plan(b, sub.data(), (int)sub.size(), t, c, &part)) return rc;
        p->parts.push_back(part);
        p->n_chunks += part->n_chunks;
    }
    *out = p.release();
    return LDPC_OK;
}

}  // namespace

extern "C" {

int ldpc_batch_create(const ldpc_code* const* codes, const ldpc_cfg* cfgs, int n_codes, int device, ldpc_batch** out) {
    if (!codes || !cfgs || !out || n_codes < 1) return fail(LDPC_ERR_INVALID_ARG, "batch: NULL argument or no codes");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(LDPC_ERR_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(LDPC_ERR_INVALID_ARG, "device %d of %d", device, ndev);
    std::unique_ptr<ldpc_batch> b(new ldpc_batch);
    b->device = device;
    CUDA_TRY(cudaSetDevice(device));
    CUDA_TRY(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device));
    for (int i = 0; i < n_codes; ++i) {
        if (!codes[i]) return fail(LDPC_ERR_INVALID_ARG, "batch: code %d is NULL", i);
        const ldpc_code& c = *codes[i];
        const ldpc_cfg& g = cfgs[i];
        if (i == 0) b->variant = g.variant;
        if (g.variant != b->variant)
            return fail(LDPC_ERR_UNSUPPORTED, "batch: code %d: every code of a batch needs the same variant", i);
        if (g.max_iter < 1 || g.max_iter > 255) return fail(LDPC_ERR_UNSUPPORTED, "batch: code %d: max_iter=%u", i, g.max_iter);
        if (g.variant == LDPC_F32_SP || g.variant == LDPC_F32_OMS) {
            if (c.mrow > ldpc::SP_MAX_L || (int)c.row_cols.size() > ldpc::SP_MAX_E || c.max_row_weight > 32 || c.z > 512)
                return fail(LDPC_ERR_UNSUPPORTED, "batch: code %d exceeds the float decoder's tables", i);
            b->codes.push_back(c);
            b->cfgs.push_back(g);
            b->beta8.push_back(std::vector<int>(c.mrow, 0));
            b->tab8.emplace_back();
            b->tab_rows.push_back(0);
            b->maxv2.push_back(0);
            b->maxf.push_back(g.max_row_metric < 1e-6f ? (float)(1.0 - (double)g.max_row_metric) : g.max_row_metric);
            continue;
        }
        if (g.variant != LDPC_INT8_OMS) return fail(LDPC_ERR_UNSUPPORTED, "batch: code %d: variant %d is not batched", i, g.variant);
        if (!(g.beta >= 0.0f && g.beta < 128.0f)) return fail(LDPC_ERR_UNSUPPORTED, "batch: code %d: beta=%g", i, g.beta);
        if (!(g.max_row_metric > -128.0f && g.max_row_metric < 128.0f))
            return fail(LDPC_ERR_UNSUPPORTED, "batch: code %d: max_row_metric=%g", i, g.max_row_metric);
        const int max8 = ldpc::max_row_i8(g.max_row_metric);
        if (max8 < 0) return fail(LDPC_ERR_UNSUPPORTED, "batch: code %d: negative row clamp", i);
        if (!ldpc::rt_dmax(c.max_row_weight) || c.z > ldpc::RT_MAX_Z || c.mrow > ldpc::RT_MAX_L ||
            (int)c.row_cols.size() > ldpc::RT_MAX_E)
            return fail(LDPC_ERR_UNSUPPORTED, "batch: code %d (Z=%d, %d layers, weight %d) exceeds the kernel's tables", i,
                        c.z, c.mrow, c.max_row_weight);
        b->codes.push_back(c);
        b->cfgs.push_back(g);
        b->beta8.push_back(std::vector<int>(c.mrow, (int)(int8_t)g.beta));
        b->tab8.emplace_back();
        b->tab_rows.push_back(0);
        b->maxv2.push_back(ldpc::half2_bits((float)max8));
        b->maxf.push_back(0.f);
    }
    *out = b.release();
    return LDPC_OK;
}

int ldpc_batch_set_offsets(ldpc_batch* b, int code, const float* beta) {
    if (!b) return fail(LDPC_ERR_INVALID_ARG, "batch is NULL");
    if (b->variant != LDPC_INT8_OMS) return fail(LDPC_ERR_UNSUPPORTED, "per-layer offsets are for int8 batches");
    if (code < 0 || code >= (int)b->codes.size()) return fail(LDPC_ERR_INVALID_ARG, "code %d of %zu", code, b->codes.size());
    std::vector<int>& v = b->beta8[code];
    for (size_t l = 0; l < v.size(); ++l) {
        const float f = beta ? beta[l] : b->cfgs[code].beta;
        if (!(f >= 0.0f && f < 128.0f)) return fail(LDPC_ERR_UNSUPPORTED, "offset %g of layer %zu outside [0, 128)", f, l);
    }
    for (size_t l = 0; l < v.size(); ++l) v[l] = (int)(int8_t)(beta ? beta[l] : b->cfgs[code].beta);
    b->tab8[code].clear();
    b->tab_rows[code] = 0;
    return LDPC_OK;
}

int ldpc_batch_set_offset_table(ldpc_batch* b, int code, const float* beta, unsigned rows) {
    if (!b) return fail(LDPC_ERR_INVALID_ARG, "batch is NULL");
    if (b->variant != LDPC_INT8_OMS) return fail(LDPC_ERR_UNSUPPORTED, "offset tables are for int8 batches");
    if (code < 0 || code >= (int)b->codes.size()) return fail(LDPC_ERR_INVALID_ARG, "code %d of %zu", code, b->codes.size());
    if (beta && (rows < 1 || rows > 255)) return fail(LDPC_ERR_INVALID_ARG, "offset table of %u rows (1..255)", rows);
    const size_t m = (size_t)b->codes[code].mrow;
    std::vector<int> tab;
    if (beta) {
        for (size_t i = 0; i < rows * m; ++i) {
            if (!(beta[i] >= 0.0f && beta[i] < 128.0f))
                return fail(LDPC_ERR_UNSUPPORTED, "offset %g of row %zu, layer %zu outside [0, 128)", beta[i], i / m, i % m);
            tab.push_back((int)(int8_t)beta[i]);
        }
    }
    b->tab8[code] = tab;
    b->tab_rows[code] = beta ? (int)rows : 0;
    std::fill(b->beta8[code].begin(), b->beta8[code].end(), (int)(int8_t)b->cfgs[code].beta);
    return LDPC_OK;
}

void ldpc_batch_destroy(ldpc_batch* b) { delete b; }

int ldpc_batch_plan_create(ldpc_batch* b, const ldpc_batch_job* jobs, int n_jobs, int threads, int cpc,
                           ldpc_batch_plan** out) {
    if (!b || !out || (n_jobs > 0 && !jobs) || n_jobs < 0) return fail(LDPC_ERR_INVALID_ARG, "batch plan: NULL argument");
    *out = nullptr;
    for (int i = 0; i < n_jobs; ++i)
        if (int rc = check_job(b, jobs[i], i)) return rc;
    CUDA_TRY(cudaSetDevice(b->device));
    int maxz = 0;
    for (int i = 0; i < n_jobs; ++i) maxz = std::max(maxz, b->codes[jobs[i].code].z);
    if (threads <= 0) threads = b->tuned_threads;
    const bool explicit_threads = threads > 0;
    if (threads <= 0) threads = std::max(256, ((maxz + 31) / 32) * 32);
    if (cpc <= 0) cpc = b->tuned_cpc > 0 ? b->tuned_cpc : 4;
    if (threads % 32 || threads > ldpc::kRtMaxThreads || threads < maxz)
        return fail(LDPC_ERR_UNSUPPORTED, "batch plan: %d threads per CTA (multiple of 32, >= Z=%d, <= %d)", threads, maxz,
                    ldpc::kRtMaxThreads);
    return plans_by_class(b, jobs, n_jobs, explicit_threads, threads, cpc, out);
}

int ldpc_batch_plan_launch(ldpc_batch_plan* p, void* stream) {
    if (!p) return fail(LDPC_ERR_INVALID_ARG, "plan is NULL");
    if (p->n_chunks == 0) return LDPC_OK;
    CUDA_TRY(cudaSetDevice(p->device));
    if (p->parts.empty()) {
        CUDA_TRY(launch_plan_kernel(p, (cudaStream_t)stream));
    } else {
        for (ldpc_batch_plan* q : p->parts)
            if (q->n_chunks) CUDA_TRY(launch_plan_kernel(q, (cudaStream_t)stream));
    }
    return LDPC_OK;
}

int ldpc_batch_plan_graph_launch(ldpc_batch_plan* p, void* stream) {
    if (!p) return fail(LDPC_ERR_INVALID_ARG, "plan is NULL");
    if (p->n_chunks == 0) return LDPC_OK;
    CUDA_TRY(cudaSetDevice(p->device));
    if (!p->exec) {
        if (!p->own) CUDA_TRY(cudaStreamCreateWithFlags(&p->own, cudaStreamNonBlocking));
        if (!p->ev_in) CUDA_TRY(cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming));
        if (!p->ev_out) CUDA_TRY(cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming));
        // per launch of the plan: a memset node (its chunk-claim counter)
        // then its kernel node; no edges between launches, so the per-class
        // launches may run side by side
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaGraphCreate(&g, 0));
        std::vector<ldpc_batch_plan*> leaves = p->parts;
        if (leaves.empty()) leaves.push_back(p);
        cudaError_t e = cudaSuccess;
        for (ldpc_batch_plan* q : leaves) {
            if (!q->n_chunks) continue;
            void* arg = q->is_float ? (void*)&q->slp : (void*)&q->lp;
            cudaKernelNodeParams kp{};
            kp.func = q->is_float ? q->kf : (void*)q->k;
            kp.gridDim = dim3((unsigned)q->grid);
            kp.blockDim = dim3((unsigned)q->threads);
            kp.sharedMemBytes = (unsigned)q->smem;
            kp.kernelParams = &arg;
            cudaMemsetParams mp;
            memset(&mp, 0, sizeof(mp));
            mp.dst = q->d_claim;
            mp.value = 0;
            mp.elementSize = sizeof(unsigned int);
            mp.width = 1;
            mp.height = 1;
            cudaGraphNode_t mnode, node;
            if ((e = cudaGraphAddMemsetNode(&mnode, g, nullptr, 0, &mp)) != cudaSuccess) break;
            if ((e = cudaGraphAddKernelNode(&node, g, &mnode, 1, &kp)) != cudaSuccess) break;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            p->exec = nullptr;
            return fail(LDPC_ERR_CUDA, "plan graph: %s", cudaGetErrorString(e));
        }
        p->graph = g;
    }
    // replay on the plan's stream, ordered after and before the caller's stream
    CUDA_TRY(cudaEventRecord(p->ev_in, (cudaStream_t)stream));
    CUDA_TRY(cudaStreamWaitEvent(p->own, p->ev_in, 0));
    CUDA_TRY(cudaGraphLaunch(p->exec, p->own));
    CUDA_TRY(cudaEventRecord(p->ev_out, p->own));
    CUDA_TRY(cudaStreamWaitEvent((cudaStream_t)stream, p->ev_out, 0));
    return LDPC_OK;
}

void ldpc_batch_plan_destroy(ldpc_batch_plan* p) { PlanDel()(p); }

int ldpc_batch_plan_kernels(const ldpc_batch_plan* p) {
    if (!p || p->n_chunks == 0) return 0;
    if (p->parts.empty()) return 1;
    int k = 0;
    for (const ldpc_batch_plan* q : p->parts) k += q->n_chunks ? 1 : 0;
    return k;
}

}  // extern "C"

namespace {
// Median of three timed launches (after a warm-up) of a plan over the jobs
// at width t and c chunks per CTA (t = 0: the batch's per-class shapes);
// *ms_out < 0 when the shape does not fit.
int time_shape(ldpc_batch* b, const ldpc_batch_job* jobs, int n_jobs, int t, int c, cudaStream_t s, cudaEvent_t e0,
               cudaEvent_t e1, double* ms_out) {
    *ms_out = -1;
    ldpc_batch_plan* p = nullptr;
    if (ldpc_batch_plan_create(b, jobs, n_jobs, t, c, &p) != LDPC_OK) return LDPC_OK;   // shape does not fit
    float ms[3] = {0, 0, 0};
    int rc = ldpc_batch_plan_launch(p, s);    // warm-up
    for (int r = 0; r < 3 && rc == LDPC_OK; ++r) {
        cudaEventRecord(e0, s);
        rc = ldpc_batch_plan_launch(p, s);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(LDPC_ERR_CUDA, "autotune: launch failed");
        else cudaEventElapsedTime(&ms[r], e0, e1);
    }
    ldpc_batch_plan_destroy(p);
    if (rc != LDPC_OK) return rc;
    std::sort(ms, ms + 3);
    *ms_out = ms[1];
    return LDPC_OK;
}

// The fastest (width, chunks per CTA) for these jobs: every width of
// kTunedWidths >= maxz and 1, 2, 4 or 8 chunks per CTA.
int tune_shape(ldpc_batch* b, const ldpc_batch_job* jobs, int n_jobs, int maxz, cudaStream_t s, cudaEvent_t e0,
               cudaEvent_t e1, int* t_out, int* c_out, double* ms_out) {
    double best = 1e30;
    int best_t = 0, best_c = 0;
    const int cpcs[] = {1, 2, 4, 8};
    for (int t : kTunedWidths) {
        if (t < maxz) continue;
        for (int c : cpcs) {
            double ms = 0;
            if (int rc = time_shape(b, jobs, n_jobs, t, c, s, e0, e1, &ms)) return rc;
            if (ms >= 0 && ms < best) {
                best = ms;
                best_t = t;
                best_c = c;
            }
        }
    }
    if (!best_t) return fail(LDPC_ERR_UNSUPPORTED, "autotune: no launch shape fits these codes");
    *t_out = best_t;
    *c_out = best_c;
    *ms_out = best;
    return LDPC_OK;
}
}  // namespace

extern "C" {

int ldpc_batch_autotune(ldpc_batch* b, const ldpc_batch_job* jobs, int n_jobs, size_t sample, int* threads_out,
                        int* cpc_out, double* ms_out) {
    if (!b || (n_jobs > 0 && !jobs) || n_jobs < 1) return fail(LDPC_ERR_INVALID_ARG, "autotune: no jobs");
    for (int i = 0; i < n_jobs; ++i)
        if (int rc = check_job(b, jobs[i], i)) return rc;
    if (sample == 0) sample = 8192;
    std::vector<ldpc_batch_job> sj(jobs, jobs + n_jobs);
    int maxz = 0;
    for (ldpc_batch_job& j : sj) {
        j.n = std::min(j.n, sample);
        j.post_out = nullptr;
        j.hard_out = nullptr;
        j.iters_out = nullptr;
        j.data_bits = nullptr;
        j.counters = nullptr;
        maxz = std::max(maxz, b->codes[j.code].z);
    }
    CUDA_TRY(cudaSetDevice(b->device));
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    int rc = LDPC_OK;
    std::vector<int> code_cls, cls_threads;
    int n_cls = 1;
    if (!getenv("LDPC_BATCH_ONE_LAUNCH") && n_jobs > 1)
        rc = plan_classes(b, sj.data(), n_jobs, false, 0, code_cls, cls_threads, &n_cls);
    double best = 1e30, worst = -1;
    int best_t = 0, best_c = 0;
    if (rc == LDPC_OK && n_cls > 1) {
        // several classes: each class is its own launch.  Candidates: every class
        // tuned on its own jobs, and one shape for all classes; the whole
        // sample plan decides between them.
        std::vector<int> ct(b->codes.size(), 0), cc(b->codes.size(), 0);
        for (int k = 0; k < n_cls && rc == LDPC_OK; ++k) {
            int kz = 0, t = 0, c = 0;
            double ms = 0;
            std::vector<ldpc_batch_job> sub = class_jobs(b, sj.data(), n_jobs, code_cls, k, &kz);
            rc = tune_shape(b, sub.data(), (int)sub.size(), kz, s, e0, e1, &t, &c, &ms);
            if (rc != LDPC_OK) break;
            for (const ldpc_batch_job& j : sub) {
                ct[j.code] = t;
                cc[j.code] = c;
            }
            if (ms > worst) {
                worst = ms;
                best_t = t;
                best_c = c;
            }
        }
        double ms_pc = -1, ms_glob = 0;
        int gt = 0, gc = 0;
        if (rc == LDPC_OK) {
            b->code_threads = ct;
            b->code_cpc = cc;
            b->tuned_threads = b->tuned_cpc = 0;
            rc = time_shape(b, sj.data(), n_jobs, 0, 0, s, e0, e1, &ms_pc);
        }
        if (rc == LDPC_OK) rc = tune_shape(b, sj.data(), n_jobs, maxz, s, e0, e1, &gt, &gc, &ms_glob);
        // third candidate: every code at its own width with the default chunks per CTA
        double ms_def = -1;
        if (rc == LDPC_OK) {
            const std::vector<int> keep_t = b->code_threads, keep_c = b->code_cpc;
            b->code_threads.clear();
            b->code_cpc.clear();
            rc = time_shape(b, sj.data(), n_jobs, 0, 0, s, e0, e1, &ms_def);
            b->code_threads = keep_t;
            b->code_cpc = keep_c;
        }
        if (rc == LDPC_OK && ms_def >= 0 && (ms_pc < 0 || ms_def <= ms_pc) && ms_def <= ms_glob) {
            b->code_threads.clear();
            b->code_cpc.clear();
            best = ms_def;
            best_t = 0;
            best_c = 0;
        } else if (rc == LDPC_OK) {
            if (ms_pc < 0 || ms_glob < ms_pc) {
                b->tuned_threads = best_t = gt;
                b->tuned_cpc = best_c = gc;
                b->code_threads.clear();
                b->code_cpc.clear();
                best = ms_glob;
            } else {
                best = ms_pc;
            }
        } else {
            b->code_threads.clear();
            b->code_cpc.clear();
        }
    } else if (rc == LDPC_OK) {
        rc = tune_shape(b, sj.data(), n_jobs, maxz, s, e0, e1, &best_t, &best_c, &best);
        // against the codes' own width with the default chunks per CTA
        double ms_def = -1;
        if (rc == LDPC_OK) {
            b->tuned_threads = b->tuned_cpc = 0;
            b->code_threads.clear();
            b->code_cpc.clear();
            rc = time_shape(b, sj.data(), n_jobs, 0, 0, s, e0, e1, &ms_def);
        }
        if (rc == LDPC_OK) {
            if (ms_def >= 0 && ms_def <= best) {
                best = ms_def;
                best_t = best_c = 0;
            } else {
                b->tuned_threads = best_t;
                b->tuned_cpc = best_c;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (rc != LDPC_OK) return rc;
    if (threads_out) *threads_out = best_t;
    if (cpc_out) *cpc_out = best_c;
    if (ms_out) *ms_out = best;
    return LDPC_OK;
}

}  // extern "C"
