// Host side of channel generation, encoding, error counting and the
// simulation driver (ldpc_generate / ldpc_encode / ldpc_llr_from_noise /
// ldpc_count_errors / ldpc_simulate).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gen.cuh"
#include "internal.h"

namespace ldpc {

namespace {
// gen_metrics.cpp:26-30, evaluated with the same float/double steps
void sigma_of(float snr, float llr_scale, float* sigma, float* sf) {
    const float three_db = 10 * log10f(2.0f);
    const float s = powf(10.0f, (float)((double)(snr + three_db) / -20.0));
    *sigma = s;
    *sf = 2 * llr_scale / (s * s);
}

// Tile shape of gen_kernel: the per-thread encoder for Z <= 64 without filler
// bits, 128 codewords per tile (halved until the tile fits 96 KB); else the
// warp encoder, 32 codewords per tile (halved until it fits 100 KB).
size_t gen_tile_shape(const GenTables& t, GenTile* tile) {
    const size_t nw = t.n / 32 + 3, dwp = t.kbits / 32 + 3;
    tile->fast = tile->clamp16 = tile->qshift = 0;
    tile->thread_enc = (t.z <= 64 && !t.any_filler) ? 1 : 0;
    size_t smem = 0;
    if (tile->thread_enc) {
        int T = 128;
        auto bytes = [&](int T_) { return (size_t)T_ * (8 * (size_t)t.mcol + 4 * (dwp + nw)); };
        while (T > 1 && bytes(T) > 96 * 1024) T /= 2;
        tile->T = T;
        smem = bytes(T);
    } else {
        int T = 32;
        const size_t warp_bytes = 4 * (size_t)(GEN_THREADS / 32) * gen_warp_words(t.kbits, t.mcol, t.z, t.n);
        auto bytes = [&](int T_) { return 4 * nw * T_ + warp_bytes; };
        while (T > 1 && bytes(T) > 100 * 1024) T /= 2;
        tile->T = T;
        smem = bytes(T);
    }
    return smem;
}

int gen_grid(ldpc_ctx* x, long long n, int* smem) {
    const GenTables& t = x->gent;
    *smem = gen_warp_words(t.kbits, t.mcol, t.z, t.n) * 4 * 8;
    const long long want = (n + 7) / 8;
    return (int)std::max<long long>(1, std::min<long long>(want, (long long)x->sms * 8));
}
}  // namespace

int setup_gen(ldpc_ctx* x) {
    const ldpc_code& c = x->code;
    GenTables& t = x->gent;
    memset(&t, 0, sizeof(t));
    // terms beyond the parameter block go to device memory; par_first is 16 bits
    if (c.mrow > GEN_MAX_PAR || (int)c.term_col.size() > 32767 || c.mcol > GEN_MAX_COLS)
        return fail(LDPC_ERR_UNSUPPORTED, "encoder schedule too large (%d parity columns, %zu terms)", c.mrow,
                    c.term_col.size());
    t.z = c.z;
    t.mcol = c.mcol;
    t.mrow = c.mrow;
    t.n = c.z * c.mcol;
    t.kbits = x->kbits;
    t.hard_words = x->hard_words;
    t.words_per_col = (c.z + 31) / 32;
    t.n_par = c.mrow;
    for (int i = 0; i < c.mrow; ++i) {
        t.par_col[i] = (int16_t)c.sched_col[i];
        t.par_first[i] = (int16_t)c.sched_first[i];
        t.par_cnt[i] = (int16_t)c.sched_cnt[i];
    }
    t.n_terms = (int)c.term_col.size();
    if (t.n_terms <= GEN_MAX_TERMS) {
        for (size_t k = 0; k < c.term_col.size(); ++k) {
            t.term_col[k] = (int16_t)c.term_col[k];
            t.term_shift[k] = (int16_t)c.term_shift[k];
        }
    } else {
        std::vector<int16_t> h(2 * (size_t)t.n_terms);
        for (int k = 0; k < t.n_terms; ++k) {
            h[k] = (int16_t)c.term_col[k];
            h[t.n_terms + k] = (int16_t)c.term_shift[k];
        }
        CUDA_TRY(cudaMalloc(&x->d_gen_terms, h.size() * sizeof(int16_t)));
        CUDA_TRY(cudaMemcpy(x->d_gen_terms, h.data(), h.size() * sizeof(int16_t), cudaMemcpyHostToDevice));
        t.term_dev = x->d_gen_terms;
    }
    t.any_punct = std::any_of(c.punct.begin(), c.punct.end(), [](uint8_t v) { return v != 0; });
    t.any_filler = std::any_of(c.filler.begin(), c.filler.end(), [](uint8_t v) { return v != 0; });
    CUDA_TRY(cudaMalloc(&x->d_masks, 2 * (size_t)t.n));
    CUDA_TRY(cudaMemcpy(x->d_masks, c.punct.data(), t.n, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(x->d_masks + t.n, c.filler.data(), t.n, cudaMemcpyHostToDevice));
    t.punct = x->d_masks;
    t.filler = x->d_masks + t.n;
    int smem = 0;
    gen_grid(x, 1, &smem);
    if (smem > 200 * 1024) return fail(LDPC_ERR_UNSUPPORTED, "generator needs %d B of shared memory", smem);
    GenTile tile;
    const size_t gsmem = gen_tile_shape(t, &tile);
    if (gsmem > 200 * 1024) return fail(LDPC_ERR_UNSUPPORTED, "generator tile needs %zu B of shared memory", gsmem);
    CUDA_TRY(allow_dynamic_smem((const void*)gen_kernel<false>, 200 * 1024));
    CUDA_TRY(allow_dynamic_smem((const void*)gen_kernel<true>, 200 * 1024));
    CUDA_TRY(allow_dynamic_smem((const void*)encode_kernel, 200 * 1024));
    return LDPC_OK;
}

void release_gen(ldpc_ctx* x) {
    cudaFree(x->d_masks);
    x->d_masks = nullptr;
    cudaFree(x->d_gen_terms);
    x->d_gen_terms = nullptr;
    cudaFree(x->d_sim_llr);
    cudaFree(x->d_sim_data);
    cudaFree(x->d_sim_hard);
    x->d_sim_llr = nullptr;
    x->d_sim_data = nullptr;
    x->d_sim_hard = nullptr;
}

int launch_gen(ldpc_ctx* x, uint64_t seed, uint64_t cw_offset, const float* snr_db, size_t n_snr, size_t n_per_snr,
               void* llr_int, float* llr_f32, uint32_t* data_bits, unsigned long long* uncoded, cudaStream_t s) {
    if (!x->code.has_enc) return fail(LDPC_ERR_INVALID_ARG, "code has no encoder table");
    if (!x->gen_ok) return fail(LDPC_ERR_UNSUPPORTED, "generator: %s", x->gen_err.c_str());
    if (n_snr < 1 || n_snr > (size_t)GEN_MAX_SNR) return fail(LDPC_ERR_INVALID_ARG, "n_snr=%zu outside 1..%d", n_snr, GEN_MAX_SNR);
    if (!snr_db) return fail(LDPC_ERR_INVALID_ARG, "snr_db is NULL");
    if (n_per_snr == 0) return LDPC_OK;
    GenJob job;
    memset(&job, 0, sizeof(job));
    job.seed = seed;
    job.cw_offset = cw_offset;
    job.n_per_snr = (long long)n_per_snr;
    job.n_snr = (int)n_snr;
    for (size_t i = 0; i < n_snr; ++i) sigma_of(snr_db[i], x->cfg.llr_scale, &job.sigma[i], &job.sigma_factor[i]);
    job.max_abs = x->cfg.max_abs_llr;
    // integer LLRs of the context's element type
    if (x->cfg.variant == LDPC_INT16_OMS) job.llr_i16 = (int16_t*)llr_int;
    else if (x->cfg.variant == LDPC_INT32_OMS) job.llr_i32 = (int32_t*)llr_int;
    else if (x->cfg.variant == LDPC_F64_SP || x->cfg.variant == LDPC_F64_OMS) job.llr_f64 = (double*)llr_int;
    else job.llr_i8 = (int8_t*)llr_int;
    job.llr_f32 = llr_f32;
    job.data_bits = data_bits;
    job.uncoded = uncoded;
    GenTile tile;
    const size_t smem = gen_tile_shape(x->gent, &tile);
    // int8 output alone, whole 4-element blocks, a clamp bound the rounding trick covers
    tile.fast = (job.llr_i8 && !job.llr_f32 && !job.llr_i16 && !job.llr_i32 && !job.llr_f64 && (x->gent.n & 3) == 0 &&
                 std::fabs(job.max_abs) < 32767.0f && n_snr <= (size_t)GEN_FAST_SNR) ? 1 : 0;
    // the 16-bit clamp after rounding needs |rx * sf| < 2^15 before the clamp: |noise| <= 9.5 (the
    // generator's largest Box-Muller radius), so |rx| <= 1 + 9.5 sigma
    tile.clamp16 = 1;
    for (size_t i = 0; i < n_snr; ++i)
        if (!((1.0 + 9.5 * (double)job.sigma[i]) * (double)job.sigma_factor[i] < 32000.0)) tile.clamp16 = 0;
    for (int r = 0; r < 10; ++r) {
        job.philox_rk[2 * r] = (uint32_t)seed + (uint32_t)r * 0x9E3779B9u;
        job.philox_rk[2 * r + 1] = (uint32_t)(seed >> 32) + (uint32_t)r * 0xBB67AE85u;
    }
    job.snr_stride = (long long)n_per_snr * x->gent.n;
    // the fast path counts uncoded errors in byte counters folded once per tile:
    // at most 255 items (4-bit blocks) per thread and tile
    // Items of 4 << qshift elements: the widest of 16, 8 and 4 that divides n and whose
    // store (4, 8 or 16 bytes at a time) the output base alignment allows.  An item adds up to
    // 1 << qshift to each byte counter: at most 256 - (1 << qshift) 4-bit blocks per thread and tile.
    const int nb = (x->gent.n + 3) / 4;
    tile.qshift = 0;
    if (tile.fast) {
        const uintptr_t al = (uintptr_t)job.llr_i8;
        for (int q = GEN_MAX_QSHIFT; q > 0; --q) {
            const int w = 4 << q;
            if (x->gent.n % w == 0 && (al % (uintptr_t)std::min(w, 16)) == 0) {
                tile.qshift = q;
                break;
            }
        }
        const long long cap = (256LL - (1LL << tile.qshift)) * GEN_THREADS;
        if (nb > cap) tile.fast = tile.qshift = 0;
        else
            while (tile.T > 1 && (long long)tile.T * nb > cap) tile.T /= 2;
    }
    const bool pf = x->gent.any_punct || x->gent.any_filler;
    const void* kfn = pf ? (const void*)gen_kernel<true> : (const void*)gen_kernel<false>;
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, GEN_THREADS, smem));
    const long long tiles = ((long long)n_per_snr + tile.T - 1) / tile.T;
    const int grid = (int)std::max<long long>(1, std::min<long long>(tiles, (long long)x->sms * std::max(per_sm, 1)));
    if (pf) gen_kernel<true><<<grid, GEN_THREADS, smem, s>>>(x->gent, job, tile);
    else gen_kernel<false><<<grid, GEN_THREADS, smem, s>>>(x->gent, job, tile);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

}  // namespace ldpc

using ldpc::fail;

extern "C" {

int ldpc_generate(ldpc_ctx* x, uint64_t seed, uint64_t cw_offset, const float* snr_db, size_t n_snr, size_t n_per_snr,
                  void* llr_int, float* llr_f32, uint32_t* data_bits, unsigned long long* uncoded, void* stream) {
    if (!x) return fail(LDPC_ERR_INVALID_ARG, "ctx is NULL");
    CUDA_TRY(cudaSetDevice(x->device));
    return ldpc::launch_gen(x, seed, cw_offset, snr_db, n_snr, n_per_snr, llr_int, llr_f32, data_bits, uncoded,
                            (cudaStream_t)stream);
}

int ldpc_encode(ldpc_ctx* x, const uint32_t* data_bits, size_t n, uint8_t* cw_bits, void* stream) {
    if (!x) return fail(LDPC_ERR_INVALID_ARG, "ctx is NULL");
    if (!x->code.has_enc) return fail(LDPC_ERR_INVALID_ARG, "code has no encoder table");
    if (!x->gen_ok) return fail(LDPC_ERR_UNSUPPORTED, "encoder: %s", x->gen_err.c_str());
    if (n == 0) return LDPC_OK;
    if (!data_bits || !cw_bits) return fail(LDPC_ERR_INVALID_ARG, "NULL buffer");
    CUDA_TRY(cudaSetDevice(x->device));
    int smem = 0;
    const int grid = ldpc::gen_grid(x, (long long)n, &smem);
    ldpc::encode_kernel<<<grid, 256, smem, (cudaStream_t)stream>>>(x->gent, data_bits, (long long)n, cw_bits);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

int ldpc_llr_from_noise(ldpc_ctx* x, const uint8_t* cw_bits, const float* noise, size_t n, float snr_db, void* llr_int,
                        float* llr_f32, unsigned long long* uncoded, void* stream) {
    if (!x) return fail(LDPC_ERR_INVALID_ARG, "ctx is NULL");
    if (!x->code.has_enc) return fail(LDPC_ERR_INVALID_ARG, "code has no encoder table (puncture/filler masks)");
    if (!x->gen_ok) return fail(LDPC_ERR_UNSUPPORTED, "generator: %s", x->gen_err.c_str());
    if (n == 0) return LDPC_OK;
    if (!cw_bits || !noise || (!llr_int && !llr_f32)) return fail(LDPC_ERR_INVALID_ARG, "NULL buffer");
    const bool is_float = x->cfg.variant == LDPC_F32_SP || x->cfg.variant == LDPC_F32_OMS;
    CUDA_TRY(cudaSetDevice(x->device));
    float sigma, sf;
    ldpc::sigma_of(snr_db, x->cfg.llr_scale, &sigma, &sf);
    const long long total = (long long)n * x->n;
    const int grid = (int)std::min<long long>((total + 255) / 256, (long long)x->sms * 16);
    ldpc::llr_from_noise_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(x->gent, cw_bits, noise, total, sigma, sf,
                                                                       x->cfg.max_abs_llr, is_float ? nullptr : llr_int,
                                                                       ldpc::llr_bytes(x->cfg.variant), llr_f32, uncoded);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

int ldpc_count_errors(ldpc_ctx* x, const uint32_t* hard, size_t n, const uint32_t* data_bits, size_t ref_period,
                      unsigned long long* counters, void* stream) {
    if (!x) return fail(LDPC_ERR_INVALID_ARG, "ctx is NULL");
    if (n == 0) return LDPC_OK;
    if (!hard || !data_bits || !counters || ref_period == 0) return fail(LDPC_ERR_INVALID_ARG, "NULL buffer or period");
    CUDA_TRY(cudaSetDevice(x->device));
    const int grid = (int)std::min<long long>(((long long)n + 7) / 8, (long long)x->sms * 8);
    ldpc::count_errors_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(hard, (long long)n, data_bits,
                                                                      (long long)ref_period, x->hard_words, x->kbits,
                                                                      x->code.z, x->code.num_par, counters);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

int ldpc_simulate(ldpc_ctx* x, uint64_t seed, uint64_t cw_offset, const float* snr_db, size_t n_snr, size_t n_per_snr,
                  ldpc_snr_stats* stats) {
    if (!x || !snr_db || !stats) return fail(LDPC_ERR_INVALID_ARG, "NULL argument");
    if (n_snr < 1 || n_snr > (size_t)ldpc::GEN_MAX_SNR) return fail(LDPC_ERR_INVALID_ARG, "n_snr=%zu", n_snr);
    CUDA_TRY(cudaSetDevice(x->device));
    const bool is_float = x->cfg.variant == LDPC_F32_SP || x->cfg.variant == LDPC_F32_OMS;
    const size_t N = (size_t)x->n, es = (size_t)ldpc::llr_bytes(x->cfg.variant);
    // chunk so that the LLRs of all SNR points fit in ~2 GB
    size_t chunk = std::max<size_t>(1, std::min<size_t>(n_per_snr, ((size_t)2 << 30) / (n_snr * N * es)));
    if (x->sim_cap < chunk * n_snr) {
        cudaFree(x->d_sim_llr);
        cudaFree(x->d_sim_data);
        cudaFree(x->d_sim_hard);
        x->d_sim_llr = x->d_sim_data = x->d_sim_hard = nullptr;
        x->sim_cap = 0;
        CUDA_TRY(cudaMalloc(&x->d_sim_llr, chunk * n_snr * N * es));
        CUDA_TRY(cudaMalloc(&x->d_sim_data, chunk * x->hard_words * 4));
        x->sim_cap = chunk * n_snr;
    }
    cudaStream_t s = x->streams[0];
    unsigned long long* dc = x->d_counters;   // [n_snr][4] decode + [n_snr] uncoded
    CUDA_TRY(cudaMemsetAsync(dc, 0, sizeof(unsigned long long) * ldpc::OMS_MAX_BUCKETS * 5, s));
    std::vector<double> ms(n_snr, 0.0);
    for (size_t off = 0; off < n_per_snr; off += chunk) {
        const size_t m = std::min(chunk, n_per_snr - off);
        int rc = ldpc::launch_gen(x, seed, cw_offset + off, snr_db, n_snr, m, is_float ? nullptr : x->d_sim_llr,
                                  is_float ? (float*)x->d_sim_llr : nullptr, (uint32_t*)x->d_sim_data,
                                  dc + ldpc::OMS_MAX_BUCKETS * 4, s);
        if (rc) return rc;
        for (size_t k = 0; k < n_snr; ++k) {
            ldpc::DecodeArgs a;
            a.llr = (const uint8_t*)x->d_sim_llr + k * m * N * es;
            a.n = m;
            a.ref_bits = (const uint32_t*)x->d_sim_data;
            a.ref_period = (long long)m;
            a.bucket_size = (long long)m;
            a.counters = dc + 4 * k;
            a.n_buckets = 1;
            CUDA_TRY(cudaEventRecord(x->ev_start, s));
            rc = ldpc::launch_decode(x, a, s);
            if (rc) return rc;
            CUDA_TRY(cudaEventRecord(x->ev_stop, s));
            CUDA_TRY(cudaEventSynchronize(x->ev_stop));
            float t = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&t, x->ev_start, x->ev_stop));
            ms[k] += t;
        }
    }
    std::vector<unsigned long long> h(ldpc::OMS_MAX_BUCKETS * 5);
    CUDA_TRY(cudaMemcpyAsync(h.data(), dc, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    for (size_t k = 0; k < n_snr; ++k) {
        stats[k].snr_db = snr_db[k];
        stats[k].codewords = h[4 * k + 0];
        stats[k].iterations = h[4 * k + 1];
        stats[k].bit_errors = h[4 * k + 2];
        stats[k].cw_errors = h[4 * k + 3];
        stats[k].uncoded_errors = h[ldpc::OMS_MAX_BUCKETS * 4 + k];
        stats[k].decode_ms = ms[k];
    }
    return LDPC_OK;
}

}  // extern "C"
