// Host side of the int8 offset min-sum decoder: kernel selection, launch geometry, launch.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "internal.h"
#include "codes_fixed.cuh"
#include "oms_f16.cuh"

namespace ldpc {

namespace {
// Shapes compiled with the check messages in registers.  Exact shapes first
// (802.11ad rate 1/2: 8 layers of weights 5,6,6,6,7,7,7,8), then padded ones.
using Shape11ad12 = FixedShape<5, 6, 6, 6, 7, 7, 7, 8>;
const int kRw11ad12[] = {5, 6, 6, 6, 7, 7, 7, 8};
#define OMS_K(S_, T_, B_) {T_, B_, oms_f16_kernel<S_, false, T_, B_>, oms_f16_kernel<S_, true, T_, B_>}
#define OMS_FIXED(S_, RW_) {S_::L, S_::D, RW_, nullptr, 0, 4, {OMS_K(S_, 640, 1), OMS_K(S_, 256, 2), OMS_K(S_, 192, 3), OMS_K(S_, 128, 5)}}
#define OMS_COMPILED(C_, RW_) {C_::L, C_::D, RW_, &kCompiled##C_, 0, 4, {OMS_K(CompiledShape<C_>, 640, 1), OMS_K(CompiledShape<C_>, 256, 2), OMS_K(CompiledShape<C_>, 192, 3), OMS_K(CompiledShape<C_>, 128, 5)}}
#define OMS_SPLIT(C_, RW_, EREG_)                                                                           \
    {C_::L, C_::D, RW_, &kCompiled##C_, C_::E - EREG_, 2,                                                    \
     {{128, 7, oms_f16_kernel<SplitShape<C_, EREG_, 128>, false, 128, 7>, oms_f16_kernel<SplitShape<C_, EREG_, 128>, true, 128, 7>}, \
      {96, 8, oms_f16_kernel<SplitShape<C_, EREG_, 96>, false, 96, 8>, oms_f16_kernel<SplitShape<C_, EREG_, 96>, true, 96, 8>}}}
#define OMS_PAD(L_, D_) {L_, D_, nullptr, nullptr, 0, 1, {{384, 1, oms_f16_kernel<PaddedShape<L_, D_>, false, 384, 1>, oms_f16_kernel<PaddedShape<L_, D_>, true, 384, 1>}}}
// compiled-in code descriptions (columns, shifts) for table matching
template <class C>
CompiledCode describe() {
    CompiledCode d;
    d.z = C::Z;
    d.L = C::L;
    d.E = C::E;
    for (int e = 0; e < C::E; ++e) {
        d.col[e] = C::col(e);
        d.shift[e] = C::shift(e);
    }
    return d;
}
const CompiledCode kCompiledCode11ad12 = describe<Code11ad12>();

const OmsInst kOmsInst[] = {
    OMS_SPLIT(Code11ad12, kRw11ad12, 30),
    OMS_COMPILED(Code11ad12, kRw11ad12),
    OMS_FIXED(Shape11ad12, kRw11ad12),
    OMS_PAD(8, 8), OMS_PAD(12, 8), OMS_PAD(8, 12), OMS_PAD(6, 16), OMS_PAD(4, 16), OMS_PAD(3, 16), OMS_PAD(4, 24),
};
#undef OMS_K
#undef OMS_FIXED
#undef OMS_COMPILED
#undef OMS_SPLIT
#undef OMS_PAD

bool matches(const OmsInst& in, const ldpc_code& c) {
    if (in.L != c.mrow) return false;
    if (in.rw) {
        for (int l = 0; l < in.L; ++l)
            if (in.rw[l] != c.row_weights[l]) return false;
        if (in.compiled) {
            // same columns; each layer's shifts = compiled shifts + one constant (mod Z)
            const CompiledCode& k = *in.compiled;
            if (k.z != c.z) return false;
            int e0 = 0;
            for (int l = 0; l < in.L; ++l) {
                const int d = c.row_weights[l];
                const int rot = ((c.row_shifts[e0] - k.shift[e0]) % c.z + c.z) % c.z;
                for (int j = 0; j < d; ++j) {
                    if (c.row_cols[e0 + j] != k.col[e0 + j]) return false;
                    if (((k.shift[e0 + j] + rot) % c.z) != c.row_shifts[e0 + j]) return false;
                }
                e0 += d;
            }
        }
        return true;
    }
    return in.D >= c.max_row_weight;
}
}  // namespace

int setup_oms(ldpc_ctx* x) {
    const ldpc_code& c = x->code;
    const int L = c.mrow;
    // LDPC_OMS_RT forces the run-time-table kernel (tuning and cross-checks);
    // per-layer offsets and offset tables need it too (the compiled shapes
    // take one offset)
    if (getenv("LDPC_OMS_RT") || !x->layer_beta8.empty() || x->tab_rows) return setup_oms_rt(x);
    const OmsInst* best = nullptr;
    const bool use_compiled = !getenv("LDPC_OMS_NO_COMPILED");
    const bool use_split = !getenv("LDPC_OMS_NO_SPLIT");
    for (const OmsInst& in : kOmsInst) {
        if (!matches(in, c) || (in.compiled && !use_compiled) || (in.smem_edges && !use_split)) continue;
        if (in.rw) { best = &in; break; }
        if (!best || in.D < best->D) best = &in;
    }
    // shapes without a register-resident instantiation: run-time tables.  The
    // padded shapes (PaddedShape<L, D>: 384-thread CTAs, one per SM) are slower
    // than the run-time-table kernel on every code that selects them (802.11ad
    // 5/8 .. 13/16, 802.11ay 13/16, 802.11n, 802.16e, G.hn: 1.14-2.48x), so they
    // run only when LDPC_OMS_PADDED asks for them; the exact and compiled
    // shapes (802.11ad 1/2) stay the default.
    if (best && !best->rw && c.z <= kRtMaxThreads && !getenv("LDPC_OMS_PADDED")) return setup_oms_rt(x);
    if (!best || L > OMS_MAX_L || L * best->D > OMS_MAX_SLOTS_E || c.z > 640) return setup_oms_rt(x);
    x->inst = best;
    x->oms_synd_loop = getenv("LDPC_OMS_SYND_LOOP") ? 1 : 0;
    OmsTables& t = x->omst;
    memset(&t, 0, sizeof(t));
    t.z = c.z;
    t.mcol = c.mcol;
    t.n = c.z * c.mcol;
    t.L = L;
    t.D = best->D;
    t.kbits = x->kbits;
    t.hard_words = x->hard_words;
    int e0 = 0;
    for (int l = 0; l < L; ++l) {
        t.rw[l] = (int16_t)c.row_weights[l];
        for (int j = 0; j < c.row_weights[l]; ++j) {
            const int slot = best->rw ? e0 + j : l * best->D + j;   // FixedShape / PaddedShape::slot
            t.colz[slot] = c.row_cols[e0 + j] * c.z;
            t.shift[slot] = (int16_t)c.row_shifts[e0 + j];
        }
        e0 += c.row_weights[l];
    }
    // groups per CTA: LDPC_OMS_G forces it (tuning); else the most groups the
    // widest compiled launch allows (<= 16: two slots per group, 32 slots)
    int G = 0;
    if (const char* e = getenv("LDPC_OMS_G")) G = atoi(e);
    const OmsLaunch* lv = nullptr;
    if (G > 0) {
        for (int i = 0; i < best->n_launch; ++i) {
            const OmsLaunch& cand = best->launch[i];
            if (((G * c.z + 31) / 32) * 32 <= cand.max_threads && (!lv || cand.max_threads < lv->max_threads)) lv = &cand;
        }
        if (!lv || G > 16) return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: %d groups of Z=%d do not fit a compiled launch", G, c.z);
    } else {
        // default: the launch whose CTA is closest to 128 threads (small CTAs keep
        // the per-layer barriers cheap; the autotuner may choose differently)
        for (int i = 0; i < best->n_launch; ++i) {
            const OmsLaunch& cand = best->launch[i];
            if (cand.max_threads < c.z) continue;
            if (!lv || std::abs(cand.max_threads - 128) < std::abs(lv->max_threads - 128)) lv = &cand;
        }
        if (!lv) lv = &best->launch[0];
        G = std::min(16, lv->max_threads / c.z);
    }
    if (G < 1) return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: Z=%d too large for the register kernel", c.z);
    x->oms_launch = lv;
    oms_fn k = x->beta0 ? lv->k_beta0 : lv->k_beta;
    // shared memory: G groups of `stride` words; stride = n rounded so that
    // stride mod 32 = ceil(32/G) (consecutive groups start in different banks)
    const int spread = (32 + G - 1) / G;
    const int stride = t.n + (((spread - t.n) % 32) + 32) % 32;
    t.G = G;
    t.stride = stride;
    x->oms_threads = ((G * c.z + 31) / 32) * 32;
    // posteriors + LLR staging + shared-memory check messages (strided by
    // the launch's maximum CTA size, a compile-time constant of the kernel)
    x->oms_smem = ((G * stride * 4 + 15) & ~15) + 2 * G * ((t.n + 15) & ~15) + best->smem_edges * lv->max_threads * 4;
    if (x->oms_smem > kOmsMaxSmem) return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: %d B of shared memory", x->oms_smem);
    CUDA_TRY(allow_dynamic_smem((const void*)k, kOmsMaxSmem));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k, x->oms_threads, x->oms_smem));
    if (per_sm < 1)
        return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: %d threads x %d B shared memory do not fit an SM",
                    x->oms_threads, x->oms_smem);
    x->oms_ctas = per_sm * x->sms;
    return LDPC_OK;
}

int launch_oms(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s) {
    if (x->oms_rt) return launch_oms_rt(x, a, s);
    if (!x->inst) return fail(LDPC_ERR_INVALID_ARG, "context was not created for the int8 decoder");
    if (a.n == 0) return LDPC_OK;
    if (a.queue < 0 || a.queue >= ldpc_ctx::kQueues) return fail(LDPC_ERR_INVALID_ARG, "queue %d", a.queue);
    OmsJob job;
    memset(&job, 0, sizeof(job));
    job.llr = (const int8_t*)a.llr;
    job.ncw = (long long)a.n;
    job.post_out = (int8_t*)a.post;
    job.hard_out = a.hard;
    job.iters_out = a.iters;
    job.ref_bits = a.ref_bits;
    job.ref_period = a.ref_period > 0 ? a.ref_period : 1;
    job.bucket_size = a.bucket_size > 0 ? a.bucket_size : (long long)a.n;
    job.counters = a.counters;
    job.n_buckets = std::max(1, std::min(a.n_buckets, OMS_MAX_BUCKETS));
    job.num_par = x->code.num_par;
    job.max_iter = (int)x->cfg.max_iter;
    job.beta2 = x->beta2;
    job.maxv2 = x->maxv2;
    job.queue = x->d_queue + a.queue;
    job.status = x->d_status;
    job.synd_loop = x->oms_synd_loop;
    const long long slots = 2LL * x->omst.G;
    const long long want = ((long long)a.n + slots - 1) / slots;
    const int grid = (int)std::min<long long>(want, x->oms_ctas);
    oms_fn k = x->beta0 ? x->oms_launch->k_beta0 : x->oms_launch->k_beta;
    k<<<grid, x->oms_threads, x->oms_smem, s>>>(x->omst, job);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

}  // namespace ldpc
