// C ABI of the B200 QC-LDPC engine (declarations: include/ldpc_b200.h):
// tables, contexts, decode entry points, host-buffer pipeline and the
// LDPCdecode_set drop-in.  Kernels live in dec_oms.cu, dec_sp.cu and gen.cu.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "internal.h"

namespace {
thread_local std::string g_err;
}

namespace ldpc {

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

uint32_t half2_bits(float v) {
    __half h = __float2half_rn(v);
    uint16_t b;
    memcpy(&b, &h, 2);
    return (uint32_t)b | ((uint32_t)b << 16);
}

}  // namespace ldpc

using ldpc::fail;

// ---------------------------------------------------------------------------
// codes
// ---------------------------------------------------------------------------
static int parse_dec(const int32_t* w, size_t nw, ldpc_code* c) {
    if (nw < 7) return fail(LDPC_ERR_BAD_TABLE, "decoder table: %zu words, need at least 7", nw);
    c->mrow = w[0];
    c->mcol = w[1];
    c->z = w[2];
    const long long ones = w[3], nf = w[5], nb = w[6];
    if (c->mrow <= 0 || c->mcol <= c->mrow || c->z <= 0 || ones <= 0 || nf < 0 || nb < 0 || c->mrow > 4096 ||
        c->mcol > 4096 || c->z > 4096 || ones > 1 << 20)
        return fail(LDPC_ERR_BAD_TABLE, "decoder table: bad header mrow=%d mcol=%d z=%d ones=%lld", c->mrow, c->mcol,
                    c->z, ones);
    const long long need = 7 + c->mrow + 2 * ones + c->mrow + 2 * nf + c->mrow + 1 + 2 * nb;
    if ((long long)nw < need)
        return fail(LDPC_ERR_BAD_TABLE, "decoder table truncated: %zu words, header promises %lld", nw, need);
    const int32_t* p = w + 7;
    c->row_weights.assign(p, p + c->mrow);
    p += c->mrow;
    c->row_cols.assign(p, p + ones);
    p += ones;
    c->row_shifts.assign(p, p + ones);
    long long sum = 0;
    c->max_row_weight = 0;
    for (int r = 0; r < c->mrow; ++r) {
        if (c->row_weights[r] < 2) return fail(LDPC_ERR_BAD_TABLE, "row %d has weight %d (< 2)", r, c->row_weights[r]);
        sum += c->row_weights[r];
        c->max_row_weight = std::max(c->max_row_weight, (int)c->row_weights[r]);
    }
    if (sum != ones) return fail(LDPC_ERR_BAD_TABLE, "row weights sum to %lld, header says %lld", sum, ones);
    for (long long e = 0; e < ones; ++e) {
        if (c->row_cols[e] < 0 || c->row_cols[e] >= c->mcol)
            return fail(LDPC_ERR_BAD_TABLE, "edge %lld: column %d outside 0..%d", e, c->row_cols[e], c->mcol - 1);
        if (c->row_shifts[e] < 0 || c->row_shifts[e] >= c->z)
            return fail(LDPC_ERR_BAD_TABLE, "edge %lld: shift %d outside 0..%d", e, c->row_shifts[e], c->z - 1);
    }
    // a column must not appear twice in a row
    int e0 = 0;
    for (int r = 0; r < c->mrow; ++r) {
        for (int j = 0; j < c->row_weights[r]; ++j)
            for (int k = 0; k < j; ++k)
                if (c->row_cols[e0 + j] == c->row_cols[e0 + k])
                    return fail(LDPC_ERR_BAD_TABLE, "row %d lists column %d twice", r, c->row_cols[e0 + j]);
        e0 += c->row_weights[r];
    }
    return LDPC_OK;
}

static int parse_enc(const int32_t* w, size_t nw, ldpc_code* c) {
    if (nw < 6) return fail(LDPC_ERR_BAD_TABLE, "encoder table: %zu words, need at least 6", nw);
    const int z = w[0], punc_cnt = w[1], fill_cnt = w[2], num_par = w[3], mrow = w[4], mcol = w[5];
    if (z != c->z || mrow != c->mrow || mcol != c->mcol)
        return fail(LDPC_ERR_BAD_TABLE, "encoder table (Z=%d %dx%d) does not match decoder table (Z=%d %dx%d)", z,
                    mrow, mcol, c->z, c->mrow, c->mcol);
    if (num_par < 1 || num_par > 16 || punc_cnt < 0 || fill_cnt < 0 || (punc_cnt & 1) || (fill_cnt & 1))
        return fail(LDPC_ERR_BAD_TABLE, "encoder table: bad num_par=%d punc=%d fill=%d", num_par, punc_cnt, fill_cnt);
    size_t pos = 6;
    if (nw < pos + 2 * (size_t)mrow) return fail(LDPC_ERR_BAD_TABLE, "encoder table truncated (counts)");
    c->par_cnts.assign(w + pos, w + pos + mrow);
    pos += mrow;
    c->par_colnum.assign(w + pos, w + pos + mrow);
    pos += mrow;
    long long sum = 0;
    for (int i = 0; i < mrow; ++i) {
        if (c->par_cnts[i] < 0 || c->par_cnts[i] > 65536) return fail(LDPC_ERR_BAD_TABLE, "bad par_cnts[%d]", i);
        if (c->par_colnum[i] < 0 || c->par_colnum[i] >= mrow) return fail(LDPC_ERR_BAD_TABLE, "bad par_colnum[%d]", i);
        sum += c->par_cnts[i];
    }
    if ((long long)nw < (long long)pos + sum + punc_cnt + fill_cnt)
        return fail(LDPC_ERR_BAD_TABLE, "encoder table truncated (offsets/lists)");
    c->par_offset.assign(w + pos, w + pos + sum);
    pos += sum;
    c->punc_list.assign(w + pos, w + pos + punc_cnt);
    pos += punc_cnt;
    c->fill_list.assign(w + pos, w + pos + fill_cnt);
    c->num_par = num_par;
    const int n = z * mcol;
    c->punct.assign(n, 0);
    c->filler.assign(n, 0);
    c->fill_cnt = 0;
    for (int pass = 0; pass < 2; ++pass) {
        const std::vector<int32_t>& lst = pass ? c->fill_list : c->punc_list;
        std::vector<uint8_t>& mask = pass ? c->filler : c->punct;
        for (size_t i = 0; i + 1 < lst.size(); i += 2) {
            if (lst[i] < 0 || lst[i + 1] >= n || lst[i] > lst[i + 1])
                return fail(LDPC_ERR_BAD_TABLE, "bad %s range %d..%d", pass ? "filler" : "puncture", lst[i], lst[i + 1]);
            // enc_fill_mask toggles the bit (encode_matrix_allocate.cpp:27-31)
            for (int b = lst[i]; b <= lst[i + 1]; ++b) mask[b] ^= 1;
            if (pass) c->fill_cnt += lst[i + 1] - lst[i] + 1;
        }
    }
    // decode par_offset (gen_encode.m:42-44,61-63): work-area byte address
    // col*16*64 + (shift%8)*2*64 + shift/8
    c->sched_col.clear();
    c->sched_first.clear();
    c->sched_cnt.clear();
    c->term_col.clear();
    c->term_shift.clear();
    size_t idx = 0;
    std::vector<uint8_t> known(mcol, 0);
    for (int k = 0; k < mcol - mrow; ++k) known[k] = 1;
    for (int i = 0; i < mrow; ++i) {
        const int pc = mcol - mrow + c->par_colnum[i];
        c->sched_col.push_back(pc);
        c->sched_first.push_back((int)c->term_col.size());
        c->sched_cnt.push_back(c->par_cnts[i]);
        for (int k = 0; k < c->par_cnts[i]; ++k, ++idx) {
            const int a = c->par_offset[idx];
            const int col = a / (16 * 64), rem = a % (16 * 64);
            const int shift = (rem % 128) * 8 + rem / 128;
            if (a < 0 || col >= mcol || shift >= z || !known[col])
                return fail(LDPC_ERR_BAD_TABLE, "encoder term %zu: address %d (column %d, shift %d) invalid", idx, a, col,
                            shift);
            c->term_col.push_back(col);
            c->term_shift.push_back(shift);
        }
        known[pc] = 1;
    }
    c->has_enc = true;
    return LDPC_OK;
}

static int read_words(const char* path, std::vector<int32_t>* out) {
    FILE* f = fopen(path, "rb");
    if (!f) return fail(LDPC_ERR_IO, "cannot open %s", path);
    std::vector<int32_t> v;
    int32_t buf[4096];
    size_t got;
    while ((got = fread(buf, 4, 4096, f)) > 0) v.insert(v.end(), buf, buf + got);
    fclose(f);
    *out = std::move(v);
    return LDPC_OK;
}

extern "C" {

const char* ldpc_last_error(void) { return g_err.c_str(); }

int ldpc_device_count(int* count) {
    if (!count) return fail(LDPC_ERR_INVALID_ARG, "count is NULL");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return LDPC_OK;
}

int ldpc_code_from_tables(const int32_t* dec_words, size_t n_dec_words, const int32_t* enc_words, size_t n_enc_words,
                          ldpc_code** out) {
    if (!out || !dec_words) return fail(LDPC_ERR_INVALID_ARG, "NULL argument");
    *out = nullptr;
    std::unique_ptr<ldpc_code> c(new ldpc_code);
    int rc = parse_dec(dec_words, n_dec_words, c.get());
    if (rc) return rc;
    if (enc_words) {
        rc = parse_enc(enc_words, n_enc_words, c.get());
        if (rc) return rc;
    }
    *out = c.release();
    return LDPC_OK;
}

int ldpc_code_load_dat(const char* enc_path, const char* dec_path, ldpc_code** out) {
    if (!out || !dec_path) return fail(LDPC_ERR_INVALID_ARG, "NULL argument");
    std::vector<int32_t> dw, ew;
    int rc = read_words(dec_path, &dw);
    if (rc) return rc;
    if (enc_path) {
        rc = read_words(enc_path, &ew);
        if (rc) return rc;
    }
    return ldpc_code_from_tables(dw.data(), dw.size(), enc_path ? ew.data() : nullptr, ew.size(), out);
}

int ldpc_code_get_info(const ldpc_code* c, ldpc_code_info* info) {
    if (!c || !info) return fail(LDPC_ERR_INVALID_ARG, "NULL argument");
    info->z = c->z;
    info->mrow = c->mrow;
    info->mcol = c->mcol;
    info->n = c->z * c->mcol;
    info->kbits = c->z * (c->mcol - c->mrow);
    info->num_par = c->num_par;
    info->fill_cnt = c->fill_cnt;
    long long e = 0;
    for (int w : c->row_weights) e += w;
    info->edges = (int)(e * c->z);
    info->max_row_weight = c->max_row_weight;
    info->hard_words = (info->kbits + 31) / 32;
    info->has_encoder = c->has_enc;
    return LDPC_OK;
}

void ldpc_code_destroy(ldpc_code* c) { delete c; }

}  // extern "C"

// ---------------------------------------------------------------------------
// contexts
// ---------------------------------------------------------------------------
namespace ldpc {

int launch_decode(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s) {
    switch (x->cfg.variant) {
        case LDPC_INT8_OMS: return launch_oms(x, a, s);
        case LDPC_INT16_OMS:
        case LDPC_INT32_OMS: return launch_int(x, a, s);
        default: return launch_sp(x, a, s);
    }
}

int8_t max_row_i8(float m) {
    // decode_row's Max_row_simd for an int8 build (decode_functions.cpp:27-32)
    if (m < 1e-6) return (int8_t)(1.0 - (double)(int8_t)m);
    return (int8_t)m;
}

}  // namespace ldpc

extern "C" {

int ldpc_ctx_create(const ldpc_code* code, const ldpc_cfg* cfg, int device, ldpc_ctx** out) {
    if (!code || !cfg || !out) return fail(LDPC_ERR_INVALID_ARG, "NULL argument");
    *out = nullptr;
    if (cfg->max_iter < 1 || cfg->max_iter > 255)
        return fail(LDPC_ERR_UNSUPPORTED, "max_iter=%u outside 1..255", cfg->max_iter);
    if (cfg->variant < LDPC_INT8_OMS || cfg->variant > LDPC_F64_OMS)
        return fail(LDPC_ERR_INVALID_ARG, "unknown variant %d", cfg->variant);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(LDPC_ERR_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(LDPC_ERR_INVALID_ARG, "device %d of %d", device, ndev);
    struct Destroy {
        void operator()(ldpc_ctx* p) const { ldpc_ctx_destroy(p); }
    };
    std::unique_ptr<ldpc_ctx, Destroy> x(new ldpc_ctx);   // a failed set-up frees what it allocated
    x->code = *code;
    x->cfg = *cfg;
    x->device = device;
    x->n = code->z * code->mcol;
    x->kbits = code->z * (code->mcol - code->mrow);
    x->hard_words = (x->kbits + 31) / 32;
    CUDA_TRY(cudaSetDevice(device));
    CUDA_TRY(cudaDeviceGetAttribute(&x->sms, cudaDevAttrMultiProcessorCount, device));
    if (cfg->variant == LDPC_INT8_OMS) {
        if (!(cfg->beta >= 0.0f && cfg->beta < 128.0f))
            return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: beta=%g outside [0, 128)", cfg->beta);
        if (!(cfg->max_row_metric > -128.0f && cfg->max_row_metric < 128.0f))
            return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: max_row_metric=%g outside int8", cfg->max_row_metric);
        const int beta8 = (int8_t)cfg->beta;
        const int max8 = ldpc::max_row_i8(cfg->max_row_metric);
        if (max8 < 0) return fail(LDPC_ERR_UNSUPPORTED, "int8 decoder: negative row clamp %d", max8);
        x->beta0 = beta8 == 0;
        x->beta2 = ldpc::half2_bits((float)beta8);
        x->maxv2 = ldpc::half2_bits((float)max8);
        int rc = ldpc::setup_oms(x.get());
        if (rc) return rc;
    } else if (cfg->variant == LDPC_INT16_OMS || cfg->variant == LDPC_INT32_OMS) {
        int rc = ldpc::setup_int(x.get());
        if (rc) return rc;
    } else {
        int rc = ldpc::setup_sp(x.get());
        if (rc) return rc;
    }
    CUDA_TRY(cudaMalloc(&x->d_queue, sizeof(unsigned long long) * ldpc_ctx::kQueues));
    CUDA_TRY(cudaMalloc(&x->d_status, sizeof(unsigned int)));
    CUDA_TRY(cudaMemset(x->d_status, 0, sizeof(unsigned int)));
    CUDA_TRY(cudaMalloc(&x->d_counters, sizeof(unsigned long long) * ldpc::OMS_MAX_BUCKETS * 5));
    for (int i = 0; i < 2; ++i) CUDA_TRY(cudaStreamCreateWithFlags(&x->streams[i], cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreate(&x->ev_start));
    CUDA_TRY(cudaEventCreate(&x->ev_stop));
    if (code->has_enc) {
        // the generator is optional: a code whose schedule it cannot hold still decodes
        x->gen_ok = ldpc::setup_gen(x.get()) == LDPC_OK;
        if (!x->gen_ok) x->gen_err = g_err;
        g_err.clear();
    }
    *out = x.release();
    return LDPC_OK;
}

}  // extern "C"

namespace {
// Rebuild an int8 context's decoder with new offsets (per layer, or a
// [rows][layer] table; both empty = cfg.beta).
int reset_offsets(ldpc_ctx* x, const std::vector<int>& layers, const std::vector<int>& tab, int rows) {
    CUDA_TRY(cudaSetDevice(x->device));
    CUDA_TRY(cudaDeviceSynchronize());   // no launch of this context may still use the old descriptor
    auto rebuild = [x](const std::vector<int>& ly, const std::vector<int>& tb, int r) {
        cudaFree(x->d_rt_code);
        cudaFree(x->d_rt_scratch);
        cudaFree(x->d_beta_tab);
        x->d_rt_code = nullptr;
        x->d_rt_scratch = nullptr;
        x->d_beta_tab = nullptr;
        x->oms_rt = false;
        x->inst = nullptr;
        x->layer_beta8 = ly;
        x->tab_beta8 = tb;
        x->tab_rows = r;
        return ldpc::setup_oms(x);
    };
    const std::vector<int> old_layers = x->layer_beta8, old_tab = x->tab_beta8;
    const int old_rows = x->tab_rows;
    const int rc = rebuild(layers, tab, rows);
    if (rc != LDPC_OK) {
        // keep the context usable with its previous offsets; report the failure
        const std::string why = ldpc_last_error();
        rebuild(old_layers, old_tab, old_rows);
        return fail(rc, "%s", why.c_str());
    }
    return LDPC_OK;
}
}  // namespace

extern "C" {

int ldpc_ctx_set_layer_offsets(ldpc_ctx* x, const float* beta) {
    if (!x) return fail(LDPC_ERR_INVALID_ARG, "ctx is NULL");
    if (x->cfg.variant != LDPC_INT8_OMS) return fail(LDPC_ERR_UNSUPPORTED, "per-layer offsets are for int8 contexts");
    std::vector<int> table;
    if (beta) {
        for (int l = 0; l < x->code.mrow; ++l) {
            if (!(beta[l] >= 0.0f && beta[l] < 128.0f))
                return fail(LDPC_ERR_UNSUPPORTED, "offset %g of layer %d outside [0, 128)", beta[l], l);
            table.push_back((int)(int8_t)beta[l]);   // truncated like cfg.beta (decode_functions.cpp:60)
        }
    }
    return reset_offsets(x, table, {}, 0);
}

int ldpc_ctx_set_offset_table(ldpc_ctx* x, const float* beta, unsigned rows) {
    if (!x) return fail(LDPC_ERR_INVALID_ARG, "ctx is NULL");
    if (x->cfg.variant != LDPC_INT8_OMS) return fail(LDPC_ERR_UNSUPPORTED, "offset tables are for int8 contexts");
    if (beta && (rows < 1 || rows > 255)) return fail(LDPC_ERR_INVALID_ARG, "offset table of %u rows (1..255)", rows);
    std::vector<int> tab;
    if (beta) {
        const size_t m = (size_t)x->code.mrow;
        for (size_t i = 0; i < rows * m; ++i) {
            if (!(beta[i] >= 0.0f && beta[i] < 128.0f))
                return fail(LDPC_ERR_UNSUPPORTED, "offset %g of row %zu, layer %zu outside [0, 128)", beta[i], i / m, i % m);
            tab.push_back((int)(int8_t)beta[i]);   // truncated like cfg.beta (decode_functions.cpp:60)
        }
    }
    return reset_offsets(x, {}, tab, beta ? (int)rows : 0);
}

void ldpc_ctx_destroy(ldpc_ctx* x) {
    if (!x) return;
    cudaSetDevice(x->device);
    cudaFree(x->d_queue);
    cudaFree(x->d_status);
    cudaFree(x->d_counters);
    cudaFree(x->d_sp_scratch);
    cudaFree(x->d_int_scratch);
    cudaFree(x->d_rt_code);
    cudaFree(x->d_rt_scratch);
    cudaFree(x->d_beta_tab);
    for (int i = 0; i < 2; ++i) {
        if (x->streams[i]) cudaStreamDestroy(x->streams[i]);
        for (int k = 0; k < 4; ++k) cudaFree(x->d_pipe[i][k]);
    }
    if (x->ev_start) cudaEventDestroy(x->ev_start);
    if (x->ev_stop) cudaEventDestroy(x->ev_stop);
    ldpc::release_gen(x);
    delete x;
}

}  // extern "C"

namespace {

// LLR element kinds of the entry points: 0 int8, 1 float, 2 int16, 3 int32, 4 double
int llr_kind(int variant) {
    switch (variant) {
        case LDPC_INT8_OMS: return 0;
        case LDPC_INT16_OMS: return 2;
        case LDPC_INT32_OMS: return 3;
        case LDPC_F64_SP:
        case LDPC_F64_OMS: return 4;
        default: return 1;
    }
}

int check_decode_args(ldpc_ctx* x, size_t n, const void* llr, int kind) {
    static const char* names[] = {"int8", "float", "int16", "int32", "double"};
    if (!x) return fail(LDPC_ERR_INVALID_ARG, "ctx is NULL");
    if (n && !llr) return fail(LDPC_ERR_INVALID_ARG, "llr is NULL");
    if (llr_kind(x->cfg.variant) != kind)
        return fail(LDPC_ERR_INVALID_ARG, "context variant %d does not take %s LLRs", x->cfg.variant, names[kind]);
    if (n > (size_t)1 << 40) return fail(LDPC_ERR_INVALID_ARG, "n=%zu too large", n);
    return LDPC_OK;
}

// Host-buffer decoding: chunks alternate between two streams; each chunk is
// copied in, decoded and copied out on its stream, so copies of one chunk
// overlap the decode of the other.
int pipe_buffer(ldpc_ctx* x, int b, int k, size_t bytes, void** out) {
    if (bytes == 0) {
        *out = nullptr;
        return LDPC_OK;
    }
    if (x->pipe_bytes[b][k] < bytes) {
        cudaFree(x->d_pipe[b][k]);
        x->d_pipe[b][k] = nullptr;
        x->pipe_bytes[b][k] = 0;
        if (cudaMalloc(&x->d_pipe[b][k], bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(LDPC_ERR_NOMEM, "device buffer of %zu bytes", bytes);
        }
        x->pipe_bytes[b][k] = bytes;
    }
    *out = x->d_pipe[b][k];
    return LDPC_OK;
}

// Host-buffer decoding: chunks alternate between two streams; each chunk is
// copied in, decoded and copied out on its stream, so the copies of one chunk
// overlap the decoding of the other.  Device buffers persist in the context.
template <class T>
int decode_host(ldpc_ctx* x, const T* llr, size_t n, T* post, uint32_t* hard, uint8_t* iters, uint64_t* tot_iter) {
    CUDA_TRY(cudaSetDevice(x->device));
    const size_t N = (size_t)x->n, HW = (size_t)x->hard_words;
    const size_t chunk = std::max<size_t>(1, std::min<size_t>(n, ((size_t)64 << 20) / (N * sizeof(T))));
    std::vector<uint8_t> it_local;
    if (tot_iter && !iters) {
        it_local.resize(n);
        iters = it_local.data();
    }
    int rc = LDPC_OK;
    for (size_t off = 0, ci = 0; rc == LDPC_OK && off < n; off += chunk, ++ci) {
        const int b = (int)(ci & 1);
        cudaStream_t s = x->streams[b];
        const size_t m = std::min(chunk, n - off);
        void *d_llr, *d_post, *d_hard, *d_it;
        if ((rc = pipe_buffer(x, b, 0, chunk * N * sizeof(T), &d_llr)) ||
            (rc = pipe_buffer(x, b, 1, post ? chunk * N * sizeof(T) : 0, &d_post)) ||
            (rc = pipe_buffer(x, b, 2, hard ? chunk * HW * 4 : 0, &d_hard)) ||
            (rc = pipe_buffer(x, b, 3, iters ? chunk : 0, &d_it)))
            break;
        if (cudaMemcpyAsync(d_llr, llr + off * N, m * N * sizeof(T), cudaMemcpyHostToDevice, s) != cudaSuccess) {
            rc = fail(LDPC_ERR_CUDA, "copy-in: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        ldpc::DecodeArgs a;
        a.llr = d_llr;
        a.n = m;
        a.post = d_post;
        a.hard = (uint32_t*)d_hard;
        a.iters = (uint8_t*)d_it;
        a.queue = b;
        rc = ldpc::launch_decode(x, a, s);
        if (rc) break;
        if ((post && cudaMemcpyAsync(post + off * N, d_post, m * N * sizeof(T), cudaMemcpyDeviceToHost, s)) ||
            (hard && cudaMemcpyAsync(hard + off * HW, d_hard, m * HW * 4, cudaMemcpyDeviceToHost, s)) ||
            (iters && cudaMemcpyAsync(iters + off, d_it, m, cudaMemcpyDeviceToHost, s))) {
            rc = fail(LDPC_ERR_CUDA, "copy-out: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
    }
    for (int b = 0; b < 2; ++b) {
        cudaError_t e = cudaStreamSynchronize(x->streams[b]);
        if (e != cudaSuccess && rc == LDPC_OK) rc = fail(LDPC_ERR_CUDA, "decode: %s", cudaGetErrorString(e));
    }
    if (rc == LDPC_OK && tot_iter) {
        uint64_t s = 0;
        for (size_t i = 0; i < n; ++i) s += iters[i];
        *tot_iter = s;
    }
    return rc;
}

}  // namespace

extern "C" {

int ldpc_decode_int8(ldpc_ctx* x, const int8_t* llr, size_t n, int8_t* post_out, uint32_t* hard_out,
                     uint8_t* iters_out, void* stream) {
    int rc = check_decode_args(x, n, llr, 0);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(x->device));
    ldpc::DecodeArgs a;
    a.llr = llr;
    a.n = n;
    a.post = post_out;
    a.hard = hard_out;
    a.iters = iters_out;
    return ldpc::launch_oms(x, a, (cudaStream_t)stream);
}

int ldpc_decode_f32(ldpc_ctx* x, const float* llr, size_t n, float* post_out, uint32_t* hard_out, uint8_t* iters_out,
                    void* stream) {
    int rc = check_decode_args(x, n, llr, 1);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(x->device));
    ldpc::DecodeArgs a;
    a.llr = llr;
    a.n = n;
    a.post = post_out;
    a.hard = hard_out;
    a.iters = iters_out;
    return ldpc::launch_sp(x, a, (cudaStream_t)stream);
}

int ldpc_decode_f64(ldpc_ctx* x, const double* llr, size_t n, double* post_out, uint32_t* hard_out, uint8_t* iters_out,
                    void* stream) {
    int rc = check_decode_args(x, n, llr, 4);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(x->device));
    ldpc::DecodeArgs a;
    a.llr = llr;
    a.n = n;
    a.post = post_out;
    a.hard = hard_out;
    a.iters = iters_out;
    return ldpc::launch_sp(x, a, (cudaStream_t)stream);
}

int ldpc_decode_count(ldpc_ctx* x, const void* llr, size_t n, uint32_t* hard_out, uint8_t* iters_out,
                      const uint32_t* data_bits, size_t ref_period, size_t bucket_size, unsigned long long* counters,
                      int n_buckets, void* stream) {
    if (!x) return fail(LDPC_ERR_INVALID_ARG, "ctx is NULL");
    if (n && !llr) return fail(LDPC_ERR_INVALID_ARG, "llr is NULL");
    if (counters && (!data_bits || ref_period == 0 || n_buckets < 1 || n_buckets > ldpc::OMS_MAX_BUCKETS))
        return fail(LDPC_ERR_INVALID_ARG, "counting needs data_bits, ref_period > 0 and 1..%d buckets",
                    ldpc::OMS_MAX_BUCKETS);
    CUDA_TRY(cudaSetDevice(x->device));
    ldpc::DecodeArgs a;
    a.llr = llr;
    a.n = n;
    a.hard = hard_out;
    a.iters = iters_out;
    a.ref_bits = counters ? data_bits : nullptr;
    a.ref_period = (long long)ref_period;
    a.bucket_size = bucket_size ? (long long)bucket_size : (long long)n;
    a.counters = counters;
    a.n_buckets = n_buckets;
    return ldpc::launch_decode(x, a, (cudaStream_t)stream);
}

int ldpc_decode_int8_host(ldpc_ctx* x, const int8_t* llr, size_t n, int8_t* post_out, uint32_t* hard_out,
                          uint8_t* iters_out, uint64_t* tot_iter) {
    int rc = check_decode_args(x, n, llr, 0);
    if (rc) return rc;
    return decode_host<int8_t>(x, llr, n, post_out, hard_out, iters_out, tot_iter);
}

int ldpc_decode_f32_host(ldpc_ctx* x, const float* llr, size_t n, float* post_out, uint32_t* hard_out,
                         uint8_t* iters_out, uint64_t* tot_iter) {
    int rc = check_decode_args(x, n, llr, 1);
    if (rc) return rc;
    return decode_host<float>(x, llr, n, post_out, hard_out, iters_out, tot_iter);
}

int ldpc_decode_f64_host(ldpc_ctx* x, const double* llr, size_t n, double* post_out, uint32_t* hard_out,
                         uint8_t* iters_out, uint64_t* tot_iter) {
    int rc = check_decode_args(x, n, llr, 4);
    if (rc) return rc;
    return decode_host<double>(x, llr, n, post_out, hard_out, iters_out, tot_iter);
}

int ldpc_decode_int16(ldpc_ctx* x, const int16_t* llr, size_t n, int16_t* post_out, uint32_t* hard_out,
                      uint8_t* iters_out, void* stream) {
    int rc = check_decode_args(x, n, llr, 2);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(x->device));
    ldpc::DecodeArgs a;
    a.llr = llr;
    a.n = n;
    a.post = post_out;
    a.hard = hard_out;
    a.iters = iters_out;
    return ldpc::launch_int(x, a, (cudaStream_t)stream);
}

int ldpc_decode_int32(ldpc_ctx* x, const int32_t* llr, size_t n, int32_t* post_out, uint32_t* hard_out,
                      uint8_t* iters_out, void* stream) {
    int rc = check_decode_args(x, n, llr, 3);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(x->device));
    ldpc::DecodeArgs a;
    a.llr = llr;
    a.n = n;
    a.post = post_out;
    a.hard = hard_out;
    a.iters = iters_out;
    return ldpc::launch_int(x, a, (cudaStream_t)stream);
}

int ldpc_decode_int16_host(ldpc_ctx* x, const int16_t* llr, size_t n, int16_t* post_out, uint32_t* hard_out,
                           uint8_t* iters_out, uint64_t* tot_iter) {
    int rc = check_decode_args(x, n, llr, 2);
    if (rc) return rc;
    return decode_host<int16_t>(x, llr, n, post_out, hard_out, iters_out, tot_iter);
}

int ldpc_decode_int32_host(ldpc_ctx* x, const int32_t* llr, size_t n, int32_t* post_out, uint32_t* hard_out,
                           uint8_t* iters_out, uint64_t* tot_iter) {
    int rc = check_decode_args(x, n, llr, 3);
    if (rc) return rc;
    return decode_host<int32_t>(x, llr, n, post_out, hard_out, iters_out, tot_iter);
}

int ldpc_decode_set_compat(ldpc_ctx* x, void* metrics, unsigned num_cw, unsigned simd_par, uint64_t* tot_iter) {
    if (!x || (!metrics && num_cw)) return fail(LDPC_ERR_INVALID_ARG, "NULL argument");
    if (simd_par == 0 || simd_par > 4096) return fail(LDPC_ERR_INVALID_ARG, "simd_par=%u", simd_par);
    const int z = x->code.z, mcol = x->code.mcol;
    const size_t spz = (z + simd_par - 1) / simd_par;
    const size_t col = (spz + 2) * simd_par;   // elements per column incl. the two pad words
    const size_t N = (size_t)x->n;
    const size_t es = (size_t)ldpc::llr_bytes(x->cfg.variant);
    std::vector<uint8_t> flat(num_cw * N * es), post(num_cw * N * es);
    uint8_t* m = (uint8_t*)metrics;
    for (size_t w = 0; w < num_cw; ++w)
        for (int c = 0; c < mcol; ++c)
            memcpy(&flat[(w * N + (size_t)c * z) * es], m + ((w * mcol + c) * col + simd_par) * es, (size_t)z * es);
    uint64_t it = 0;
    int rc;
    switch (llr_kind(x->cfg.variant)) {
        case 0: rc = decode_host<int8_t>(x, (const int8_t*)flat.data(), num_cw, (int8_t*)post.data(), nullptr, nullptr, &it); break;
        case 2: rc = decode_host<int16_t>(x, (const int16_t*)flat.data(), num_cw, (int16_t*)post.data(), nullptr, nullptr, &it); break;
        case 3: rc = decode_host<int32_t>(x, (const int32_t*)flat.data(), num_cw, (int32_t*)post.data(), nullptr, nullptr, &it); break;
        case 4: rc = decode_host<double>(x, (const double*)flat.data(), num_cw, (double*)post.data(), nullptr, nullptr, &it); break;
        default: rc = decode_host<float>(x, (const float*)flat.data(), num_cw, (float*)post.data(), nullptr, nullptr, &it);
    }
    if (rc) return rc;
    for (size_t w = 0; w < num_cw; ++w)
        for (int c = 0; c < mcol; ++c)
            memcpy(m + ((w * mcol + c) * col + simd_par) * es, &post[(w * N + (size_t)c * z) * es], (size_t)z * es);
    if (tot_iter) *tot_iter = it;
    return LDPC_OK;
}

}  // extern "C"
